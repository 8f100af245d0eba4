// Host side of libglu_b200: handles, schedule planning and the C ABI.
//
// One handle replaces the per-call work of LUonDevice (src/numeric.cu:347-639):
// the pattern is uploaded once, the level sets are built on the GPU, and the
// factorization schedule is planned once; every factorization then only
// enqueues kernels on the caller's stream (no allocation, no per-level host
// synchronization, numeric.cu:615-616).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "glu_internal.h"
#include "glu_kernels.h"

namespace glu {

static thread_local std::string g_last_error;

Status set_error(Status s, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return s;
}

static Status cuda_fail(cudaError_t e, const char *what) {
    return set_error(e == cudaErrorMemoryAllocation ? GLU_ERR_NOMEM : GLU_ERR_CUDA, "%s: %s", what,
                     cudaGetErrorString(e));
}

#define GLU_CUDA(call, what)                                  \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(e_, (what));  \
    } while (0)

// An NVTX range around a public call: the calls appear by name on a profiler
// timeline (Nsight Systems, ncu's NVTX filters); without a tool attached the
// push and pop return at once.
struct TraceRange {
    explicit TraceRange(const char *name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
};

// Device allocations still to fail (GLU_INJECT_ALLOC_FAILURES).
static std::atomic<int> g_fail_allocs{0};

// Bytes of supernode-update position tables held by all handles, per device
// (their sum is kept under a quarter of the device's memory).
constexpr int kMaxDevices = 64;
static std::atomic<uint64_t> g_pos_bytes[kMaxDevices];

static bool injected_alloc_failure() {
    int v = g_fail_allocs.load(std::memory_order_relaxed);
    while (v > 0)
        if (g_fail_allocs.compare_exchange_weak(v, v - 1, std::memory_order_relaxed)) return true;
    return false;
}

// Device buffer owned by a handle.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t alloc(size_t b) {
        release();
        if (b == 0) return cudaSuccess;
        if (injected_alloc_failure()) return cudaErrorMemoryAllocation;
        cudaError_t e = cudaMalloc(&p, b);
        if (e == cudaSuccess) bytes = b;
        return e;
    }
    cudaError_t ensure(size_t b) { return b <= bytes ? cudaSuccess : alloc(b); }
    template <class T>
    T *as() const { return static_cast<T *>(p); }
};

template <class T>
static cudaError_t upload(DevBuf &d, const std::vector<T> &h) {
    cudaError_t e = d.alloc(sizeof(T) * std::max<size_t>(h.size(), 1));
    if (e != cudaSuccess || h.empty()) return e;
    return cudaMemcpy(d.p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
}

// Kernel kinds of glu_factor for the optional per-kernel profile.
enum KernelKind {
    KK_PERT = 0, KK_LEVEL, KK_CHAIN, KK_SCALE, KK_DGATHER, KK_PANEL, KK_UPDATE, KK_DSCATTER, KK_CHECK,
    KK_SN_DIAG, KK_SN_PANEL, KK_SN_UPDATE, KK_PACK, KK_UPDATE_TC, KK_DIAG_INV, KK_COUPLE_PACK
};
static const char *const kKindNames[GLU_KERNEL_KINDS] = {
    "k_colsum+k_pert_finish", "k_factor_level", "k_factor_chain", "k_scale_level", "k_dense_gather",
    "k_dense_panel", "k_dense_update", "k_dense_scatter", "k_check_pivots", "k_sn_diag", "k_sn_panel",
    "k_sn_update", "k_dense_pack", "k_dense_update_tc", "k_dense_diag_inv", "k_couple_pack"};

// Events around every launch of one glu_factor call, when enabled.
struct KernelProfiler {
    bool on = false;
    std::vector<cudaEvent_t> ev;
    std::vector<int> kind;
    size_t used = 0;
    float ms[GLU_KERNEL_KINDS] = {};
    uint32_t n[GLU_KERNEL_KINDS] = {};
    cudaError_t begin(cudaStream_t st) {
        if (!on) return cudaSuccess;
        while (ev.size() < 2 * (used + 1)) {
            cudaEvent_t e;
            cudaError_t r = cudaEventCreate(&e);
            if (r != cudaSuccess) return r;
            ev.push_back(e);
        }
        return cudaEventRecord(ev[2 * used], st);
    }
    cudaError_t end(int k, cudaStream_t st) {
        if (!on) return cudaSuccess;
        if (kind.size() < used + 1) kind.resize(used + 1);
        kind[used] = k;
        cudaError_t r = cudaEventRecord(ev[2 * used + 1], st);
        ++used;
        return r;
    }
    void collect() {
        if (!on) return;
        for (int k = 0; k < GLU_KERNEL_KINDS; ++k) {
            ms[k] = 0;
            n[k] = 0;
        }
        for (size_t i = 0; i < used; ++i) {
            float t = 0;
            cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]);
            ms[kind[i]] += t;
            n[kind[i]]++;
        }
        used = 0;
    }
    ~KernelProfiler() {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
};

enum StepKind { STEP_LEVEL = 0, STEP_CHAIN = 1 };
// One level of the supernodal schedule: supernodes [i0, i1) of the level order.
struct SnLevel {
    uint32_t i0, i1;        // supernodes (level order)
    uint32_t pb0, pblocks;  // blocks in the panel map
    uint32_t ub0, ublocks;  // tiles in the update map
    uint32_t db0, dblocks;  // blocks in the diagonal-block map (supernodes of width >= 2)
    uint32_t atomic;
    uint32_t panel_w;       // widest supernode with a block of its own in the panel map
};
struct Step {
    int kind;
    uint32_t l0, l1;  // sparse levels [l0, l1)
};
struct CoupleGroup {
    uint32_t c0, c1;  // deferred columns [c0, c1) (slots)
};

}  // namespace glu

using namespace glu;

struct glu_symbolic_s {
    SymbolicData s;
};

struct glu_handle_s {
    int device = 0;
    uint32_t n = 0, nnz = 0, batch = 1;
    SymbolicData pat;  // host copy of the pattern (csr_pos included)
    DevBuf d_cptr, d_ridx, d_diag, d_rptr, d_cidx, d_rdiag, d_cpos;
    DevPattern P{};
    DevBuf d_val;
    // levels
    int32_t num_lev = 0;
    std::vector<int32_t> level_ptr, level_idx;
    // factor plan
    glu_tuning tune{};
    uint32_t t = 0, m = 0;
    bool dense_buffer = false;  // tail factored in d_dense (not in place)
    std::vector<uint32_t> doff_h, tail_start_h;
    DevBuf d_doff, d_tail_start, d_dense, d_sched, d_item_off, d_levels;
    std::vector<LevelInfo> levels_h;
    std::vector<uint32_t> items_h;
    std::vector<uint64_t> work_h;
    std::vector<Step> steps;
    uint32_t chain_cluster = 8;
    FactorPlanDev F{};
    double flops = 0;
    // supernodal plan of the sparse part (used when tune.sn_width != 0)
    bool use_sn = false;
    uint32_t nsn = 0;
    DevBuf d_sn_meta, d_sn_dmap, d_sn_dsmall, d_sn_pmap, d_sn_umap, d_sn_psmall, d_sn_usmall, d_sn_tgt_off, d_sn_tgt, d_sn_pos, d_sn_pos_off;
    uint64_t pos_bytes = 0;  // bytes of d_sn_pos counted in g_pos_bytes
    std::vector<SnLevel> sn_levels;
    SnPlanDev SN{};
    // deferred coupling of the sparse part into the dense tail: per supernode
    // its cut, per deferred column and 128-wide tail block the CSC range of
    // its tail rows and the CSR range of its tail columns there, the groups
    // of up to 128 columns
    DevBuf d_sn_cut, d_couple_lstart, d_couple_ustart;
    std::vector<CoupleGroup> couple_groups;
    uint32_t couple_cols = 0;
    DevBuf d_ss_map[2], d_ss_meta[2], d_ss_small[2];  // supernodal L and U sweeps
    DevBuf d_ss_woff[2], d_ss_widx[2], d_ss_roff[2], d_ss_ridx[2], d_ss_indeg[2];  // their fused form
    DevBuf d_sweep_done;  // per value set and supernode: releases received (fused sweeps)
    std::vector<SnSweepLevel> ss_levels[2];
    // solve plan
    DevBuf d_sw_cols[4], d_sw_lptr[4], d_sw_ioff[4], d_tail_row_start, d_xo;
    std::vector<SweepStep> sw_steps[4];
    SolvePlanDev S{};
    // transforms (forward in/out, transposed in/out)
    DevBuf d_tr[8];
    TransformDev T{};
    bool has_transform = false;
    // source matrix A0
    bool has_source = false;
    uint32_t nnz_src = 0;
    DevBuf d_src_lu, d_src_scale, d_a0_rptr, d_a0_cidx, d_a0_vmap, d_a0_cptr, d_a0_ridx, d_a0_ident, d_ax0;
    bool ax0_loaded = false;
    // work buffers
    DevBuf d_status, d_pert, d_colmax, d_diag_scratch, d_counters, d_ticket, d_flags, d_y, d_io32, d_b64,
        d_x64, d_r64, d_norms;
    uint32_t *h_status = nullptr;  // pinned
    double *h_norms = nullptr;     // pinned
    size_t h_norms_cap = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // dense tail look-ahead: high-priority stream for the panels, fork /
    // panel-done / rest-done events
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_panel = nullptr, ev_rest = nullptr;
    // tensor-core dense update: BF16 three-part operand packs and their TMA maps
    // (allocated on the first factorization that uses them)
    DevBuf d_packA, d_packB, d_tc_counter;
    // inverses of the dense tail's 64 x 64 diagonal blocks (L and U) per value
    // set, for the dense triangular solves
    DevBuf d_dinv;
    CUtensorMap map_packA{}, map_packB{};
    uint32_t pack_m = 0;
    uint32_t num_sms = 148;
    uint32_t spin_limit = kSpinLimit;
    bool inject_unset_flag = false;  // GLU_INJECT_UNSET_SOLVE_FLAG, for the next solve
    // statistics of a factorization enqueued and not yet finished
    uint64_t pending_launches = 0;
    double pending_upd_bytes = 0, pending_upd_flops = 0;
    KernelProfiler prof;
    bool factored = false;
    glu_stats stats{};

    ~glu_handle_s() {
        if (pos_bytes && device >= 0 && device < kMaxDevices) g_pos_bytes[device] -= pos_bytes;
        if (h_status) cudaFreeHost(h_status);
        if (h_norms) cudaFreeHost(h_norms);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_panel) cudaEventDestroy(ev_panel);
        if (ev_rest) cudaEventDestroy(ev_rest);
        if (aux) cudaStreamDestroy(aux);
    }
};

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

inline cudaStream_t S_(glu_stream s) { return static_cast<cudaStream_t>(s); }

// Largest trailing block [t, n) in which every entry is in the pattern.
void find_full_tail(const SymbolicData &s, uint32_t min_m, uint32_t &t, uint32_t &m) {
    const uint32_t n = s.n;
    // run[j]: first row of the contiguous run of rows ending at n-1 in column j
    std::vector<uint32_t> run(n);
    for (uint32_t j = 0; j < n; ++j) {
        uint32_t a = s.sym_c_ptr[j], b = s.sym_c_ptr[j + 1];
        if (b == a || s.sym_r_idx[b - 1] != n - 1) {
            run[j] = n;
            continue;
        }
        uint32_t p = b - 1;
        while (p > a && s.sym_r_idx[p - 1] == s.sym_r_idx[p] - 1) --p;
        run[j] = s.sym_r_idx[p];
    }
    uint32_t best = n, mx = 0;
    for (uint32_t c = n; c-- > 0;) {
        mx = std::max(mx, run[c]);
        if (mx <= c)
            best = c;
        else
            break;
    }
    t = best;
    m = n - best;
    if (m < min_m || m == 0) {
        t = n;
        m = 0;
    }
}

// Cost model of the split point t: the columns [t, n) are factored as a dense
// block, the columns in front of t level by level.  Dense: 2/3 m^3 flops at
// kDenseRate plus kPanelLatency per panel step.  Sparse: the update work of
// the columns < t at kSparseRate plus kLevelLatency per level that still has
// an active column < t.  Returns the t of least estimated time with
// m <= max_m (t = n: no dense tail).
constexpr double kDenseRate = 30e12, kDenseRateTc = 120e12, kPanelLatency = 20e-6;
// Default width from which trailing blocks factor with panel look-ahead.
constexpr uint32_t kLookaheadMin = 3072;
// Default width from which trailing blocks update on the tensor cores.
constexpr uint32_t kDenseTcMin = 1024;
// Cost of one deferred coupling product (up to 128 columns over the whole
// m x m dense block), in scattered supernode-update entries per entry of the
// block.
constexpr double kCoupleGroupCost = 0.25;
constexpr double kSparseRate = 0.2e12, kLevelLatency = 8e-6;

uint32_t choose_split(const SymbolicData &s, const std::vector<int32_t> &level_ptr,
                      const std::vector<int32_t> &level_idx, uint32_t max_m, const glu_tuning &tu) {
    const uint32_t n = s.n;
    // sparse work of column k and the first column of each level
    std::vector<double> pre(n + 1, 0.0);
    for (uint32_t k = 0; k < n; ++k) {
        double L = s.sym_c_ptr[k + 1] - s.l_col_ptr[k] - 1;
        double U = s.csr_r_ptr[k + 1] - s.csr_diag_ptr[k] - 1;
        pre[k + 1] = pre[k] + L + 2 * L * U;
    }
    std::vector<uint32_t> lev_first;
    for (size_t l = 0; l + 1 < level_ptr.size(); ++l) {
        uint32_t first = n;
        for (int32_t q = level_ptr[l]; q < level_ptr[l + 1]; ++q) {
            uint32_t k = uint32_t(level_idx[q]);
            if (s.l_col_ptr[k] + 1 != s.sym_c_ptr[k + 1]) {
                first = k;  // ascending within a level
                break;
            }
        }
        if (first < n) lev_first.push_back(first);
    }
    std::sort(lev_first.begin(), lev_first.end());
    double best = 1e300;
    uint32_t best_t = n;
    const int64_t lo = max_m >= n ? 0 : int64_t(n) - max_m;
    for (int64_t tt = n; tt >= lo; tt -= 16) {
        const uint32_t t = uint32_t(tt);
        double m = double(n - t);
        const double rate = tu.dense_rate ? 1e9 * tu.dense_rate
                                          : (tu.dense_tc_min && m >= tu.dense_tc_min ? kDenseRateTc : kDenseRate);
        double dense = m > 0 ? (2.0 / 3.0) * m * m * m / rate + std::ceil(m / kDenseNB) * kPanelLatency : 0;
        double nlev = double(std::lower_bound(lev_first.begin(), lev_first.end(), t) - lev_first.begin());
        double sparse = pre[t] / kSparseRate + nlev * kLevelLatency;
        if (dense + sparse < best) {
            best = dense + sparse;
            best_t = t;
        }
    }
    return best_t;
}

// Level schedule of one sparse sweep over the columns [0, t) (tail columns are
// solved before or after it densely).  Dependencies:
//   L  (forward, scatter):  j needs c < j with L(j,c) != 0  (CSR row j left of diag)
//   U  (backward, scatter): j needs c > j with U(j,c) != 0  (CSR row j right of diag)
//   U^T (forward, gather):  j needs i < j with U(i,j) != 0  (CSC column j above diag)
//   L^T (backward, gather): j needs i > j with L(i,j) != 0  (CSC column j below diag)
// Work items of pivot j: its entries in chunks of kSweepChunk (at least one,
// the dividing sweeps store x_j).  Levels with more than `thin` items get
// their own launch; runs of thinner levels go to the cluster kernel.
void build_sweep(const SymbolicData &s, uint32_t t, int mode, uint32_t thin, std::vector<uint32_t> &cols,
                 std::vector<uint32_t> &lptr, std::vector<uint32_t> &item_off, std::vector<SweepStep> &steps) {
    std::vector<int32_t> lev(t, 0);
    int32_t nlev = 0;
    const bool forward = (mode == SWEEP_L || mode == SWEEP_UT);
    for (uint32_t q = 0; q < t; ++q) {
        const uint32_t j = forward ? q : t - 1 - q;
        int32_t mx = -1;
        if (mode == SWEEP_L) {
            for (uint32_t e = s.csr_r_ptr[j]; e < s.csr_diag_ptr[j]; ++e) mx = std::max(mx, lev[s.csr_c_idx[e]]);
        } else if (mode == SWEEP_U) {
            for (uint32_t e = s.csr_diag_ptr[j] + 1; e < s.csr_r_ptr[j + 1]; ++e) {
                uint32_t c = s.csr_c_idx[e];
                if (c < t) mx = std::max(mx, lev[c]);
            }
        } else if (mode == SWEEP_UT) {
            for (uint32_t p = s.sym_c_ptr[j]; p < s.l_col_ptr[j]; ++p) mx = std::max(mx, lev[s.sym_r_idx[p]]);
        } else {
            for (uint32_t p = s.l_col_ptr[j] + 1; p < s.sym_c_ptr[j + 1]; ++p) {
                uint32_t i = s.sym_r_idx[p];
                if (i < t) mx = std::max(mx, lev[i]);
            }
        }
        lev[j] = mx + 1;
        nlev = std::max(nlev, mx + 2);
    }
    lptr.assign(size_t(nlev) + 1, 0);
    for (uint32_t j = 0; j < t; ++j) lptr[lev[j] + 1]++;
    for (int32_t l = 0; l < nlev; ++l) lptr[l + 1] += lptr[l];
    cols.assign(t, 0);
    {
        std::vector<uint32_t> cur(lptr.begin(), lptr.end() - 1);
        for (uint32_t j = 0; j < t; ++j) cols[cur[lev[j]]++] = j;
    }
    item_off.assign(size_t(t) + 1, 0);
    for (uint32_t q = 0; q < t; ++q) {
        const uint32_t j = cols[q];
        uint32_t len;
        if (mode == SWEEP_L)
            len = s.sym_c_ptr[j + 1] - s.l_col_ptr[j] - 1;
        else if (mode == SWEEP_U)
            len = s.l_col_ptr[j] - s.sym_c_ptr[j];
        else if (mode == SWEEP_UT)
            len = s.csr_r_ptr[j + 1] - s.csr_diag_ptr[j] - 1;
        else
            len = s.csr_diag_ptr[j] - s.csr_r_ptr[j];
        item_off[q + 1] = item_off[q] + std::max<uint32_t>(1, (len + kSweepChunk - 1) / kSweepChunk);
    }
    auto items = [&](int32_t l) { return item_off[lptr[l + 1]] - item_off[lptr[l]]; };
    steps.clear();
    int32_t l = 0;
    while (l < nlev) {
        if (items(l) > thin) {
            steps.push_back(SweepStep{0, uint32_t(l), uint32_t(l + 1), lptr[l], lptr[l + 1]});
            ++l;
        } else {
            int32_t e = l;
            while (e < nlev && items(e) <= thin) ++e;
            steps.push_back(SweepStep{1, uint32_t(l), uint32_t(e), lptr[l], lptr[e]});
            l = e;
        }
    }
}

uint32_t pick_group(double avg_l, uint32_t forced) {
    if (forced) return forced;
    if (avg_l <= 6) return 4;
    if (avg_l <= 12) return 8;
    if (avg_l <= 24) return 16;
    return 32;
}

// Supernodal schedule of the sparse columns [0, t).  Column k joins the
// supernode [s0, k) when k - s0 < width, Lpat(k-1) = {k} u Lpat(k), and the
// rows s0..k-1 of column k are all present (dense diagonal block).  A
// supernode's level is one more than the largest level among the supernodes
// holding its columns' dependencies (symbolic.cc:106-151: U(c',c) != 0 with
// Lpat(c') nonempty, and L(c,c') != 0).
Status build_sn_plan(glu_handle_s *h) {
    const SymbolicData &s = h->pat;
    const uint32_t t = h->t;
    const uint32_t width = std::min<uint32_t>(h->tune.sn_width, kSnMaxWidth);
    h->use_sn = width > 0 && t > 0;
    h->nsn = 0;
    h->sn_levels.clear();
    h->couple_groups.clear();
    h->couple_cols = 0;
    h->stats.sn_update_flops = h->stats.sn_update_bytes = h->stats.sn_panel_bytes = 0;
    h->S.sn[0] = SnSweepPlan{};
    h->S.sn[1] = SnSweepPlan{};
    h->stats.sn_sweep_levels = 0;
    if (!h->use_sn) return GLU_OK;
    auto nl = [&](uint32_t c) { return s.sym_c_ptr[c + 1] - s.l_col_ptr[c] - 1; };
    auto nu = [&](uint32_t c) { return s.csr_r_ptr[c + 1] - s.csr_diag_ptr[c] - 1; };
    std::vector<uint32_t> first(1, 0);
    for (uint32_t k = 1, s0 = 0; k < t; ++k) {
        bool join = k - s0 < width && nl(k - 1) == nl(k) + 1 && s.sym_r_idx[s.l_col_ptr[k - 1] + 1] == k &&
                    s.l_col_ptr[k] >= s.sym_c_ptr[k] + (k - s0) && s.sym_r_idx[s.l_col_ptr[k] - (k - s0)] == s0;
        if (join)
            join = std::equal(s.sym_r_idx.begin() + s.l_col_ptr[k - 1] + 2, s.sym_r_idx.begin() + s.sym_c_ptr[k],
                              s.sym_r_idx.begin() + s.l_col_ptr[k] + 1);
        if (!join) {
            first.push_back(k);
            s0 = k;
        }
    }
    const uint32_t ns = uint32_t(first.size());
    first.push_back(t);
    std::vector<uint32_t> sn_of(t);
    for (uint32_t q = 0; q < ns; ++q)
        for (uint32_t c = first[q]; c < first[q + 1]; ++c) sn_of[c] = q;
    std::vector<int32_t> lev(ns, 0);
    int32_t nlev = 0;
    for (uint32_t q = 0; q < ns; ++q) {
        const uint32_t s0 = first[q];
        int32_t mx = -1;
        for (uint32_t c = s0; c < first[q + 1]; ++c) {
            for (uint32_t p = s.sym_c_ptr[c]; p < s.l_col_ptr[c]; ++p) {
                const uint32_t r = s.sym_r_idx[p];
                if (r < s0 && nl(r) > 0) mx = std::max(mx, lev[sn_of[r]]);
            }
            for (uint32_t e = s.csr_r_ptr[c]; e < s.csr_diag_ptr[c]; ++e) {
                const uint32_t c2 = s.csr_c_idx[e];
                if (c2 < s0) mx = std::max(mx, lev[sn_of[c2]]);
            }
        }
        lev[q] = mx + 1;
        nlev = std::max(nlev, mx + 2);
    }
    // level order (ascending column within a level)
    std::vector<uint32_t> lcount(size_t(nlev) + 1, 0);
    for (uint32_t q = 0; q < ns; ++q) lcount[lev[q] + 1]++;
    for (int32_t l = 0; l < nlev; ++l) lcount[l + 1] += lcount[l];
    std::vector<uint32_t> order(ns);
    {
        std::vector<uint32_t> cur(lcount.begin(), lcount.end() - 1);
        for (uint32_t q = 0; q < ns; ++q) order[cur[lev[q]]++] = q;
    }
    // Deferred coupling: supernode q's update of the dense tail is the corner
    // of its L21 rows >= t (a suffix of a rows) by its targets >= t (a suffix
    // of b).  When the tail updates on the tensor cores, the supernodes with
    // the largest corners per column leave theirs to tensor-core products
    // after the sparse part, up to 128 columns each.  A product costs about
    // kCoupleGroupCost m^2 scattered entry updates (the whole block's C read
    // and written, the MMAs), divided by tune.defer_tail; the prefix of
    // supernodes, by corner area per column, that saves most is taken.
    std::vector<uint32_t> ca(ns, 0), cb(ns, 0);
    std::vector<uint8_t> deferred(ns, 0);
    const bool tc_tail = h->m && h->tune.dense_tc_min && h->m >= h->tune.dense_tc_min;
    if (tc_tail && h->tune.defer_tail) {
        std::vector<std::pair<double, uint32_t>> cand;
        for (uint32_t q = 0; q < ns; ++q) {
            const uint32_t w = first[q + 1] - first[q], last = first[q + 1] - 1;
            const uint32_t *r0 = s.sym_r_idx.data() + s.l_col_ptr[last] + 1, *r1 = s.sym_r_idx.data() + s.sym_c_ptr[last + 1];
            const uint32_t *c0 = s.csr_c_idx.data() + s.csr_diag_ptr[last] + 1, *c1 = s.csr_c_idx.data() + s.csr_r_ptr[last + 1];
            ca[q] = uint32_t(r1 - std::lower_bound(r0, r1, t));
            cb[q] = uint32_t(c1 - std::lower_bound(c0, c1, t));
            const bool small = h->tune.sn_small && w <= kSnSmallWidth && (r1 - r0) <= 32 && (c1 - c0) <= 32;
            if (!small && ca[q] && cb[q]) cand.push_back({double(ca[q]) * cb[q] / w, q});
        }
        std::sort(cand.begin(), cand.end(), [](const auto &x, const auto &y) {
            return x.first != y.first ? x.first > y.first : x.second < y.second;
        });
        const double group_cost = kCoupleGroupCost * double(h->m) * h->m / h->tune.defer_tail;
        double saved = 0, best = 0;
        uint64_t cols = 0;
        size_t take = 0;
        for (size_t c = 0; c < cand.size(); ++c) {
            const uint32_t q = cand[c].second;
            cols += first[q + 1] - first[q];
            saved += double(ca[q]) * cb[q];
            const double gain = saved - double((cols + kTcTile - 1) / kTcTile) * group_cost;
            if (gain > best) {
                best = gain;
                take = c + 1;
            }
        }
        for (size_t c = 0; c < take; ++c) deferred[cand[c].second] = 1;
        if (take) {
            // deferred columns ascending; per slot and 128-wide tail block the
            // CSC positions of its tail rows and the CSR positions of its tail
            // columns that fall in the block
            std::vector<uint32_t> kcols;
            for (uint32_t q = 0; q < ns; ++q)
                if (deferred[q])
                    for (uint32_t k = first[q]; k < first[q + 1]; ++k) kcols.push_back(k);
            const uint32_t nblk = (h->m + kTcTile - 1) / kTcTile;
            std::vector<uint32_t> lstart(kcols.size() * (nblk + 1)), ustart(kcols.size() * (nblk + 1));
            for (size_t g = 0; g < kcols.size(); ++g) {
                const uint32_t k = kcols[g];
                const uint32_t *r0 = s.sym_r_idx.data() + s.sym_c_ptr[k], *r1 = s.sym_r_idx.data() + s.sym_c_ptr[k + 1];
                const uint32_t *c0 = s.csr_c_idx.data() + s.csr_r_ptr[k], *c1 = s.csr_c_idx.data() + s.csr_r_ptr[k + 1];
                for (uint32_t b = 0; b <= nblk; ++b) {
                    const uint32_t key = t + std::min<uint32_t>(b * kTcTile, h->m);
                    lstart[g * (nblk + 1) + b] = uint32_t(std::lower_bound(r0, r1, key) - s.sym_r_idx.data());
                    ustart[g * (nblk + 1) + b] = uint32_t(std::lower_bound(c0, c1, key) - s.csr_c_idx.data());
                }
            }
            for (uint32_t c0 = 0; c0 < kcols.size(); c0 += kTcTile)
                h->couple_groups.push_back(CoupleGroup{c0, std::min<uint32_t>(uint32_t(kcols.size()), c0 + kTcTile)});
            h->couple_cols = uint32_t(kcols.size());
            GLU_CUDA(upload(h->d_couple_lstart, lstart), "upload coupling plan");
            GLU_CUDA(upload(h->d_couple_ustart, ustart), "upload coupling plan");
        }
    }
    std::vector<uint2> cut(ns);
    std::vector<uint4> meta(ns);
    std::vector<uint2> pmap, umap;
    std::vector<uint32_t> psmall, usmall, dsmall, tgt(size_t(ns) + 1, 0);
    std::vector<uint2> dmap;
    std::vector<uint64_t> pos_off(size_t(ns) + 1, 0);
    const uint32_t PT = kSnPanelThreads, UT = 64, TW = kSnPanelThreads / 32;
    double upd_flops = 0, upd_bytes = 0, pan_bytes = 0;
    for (int32_t l = 0; l < nlev; ++l) {
        uint32_t updating = 0, panel_w = 0;
        const uint32_t pb0 = uint32_t(pmap.size()), ub0 = uint32_t(umap.size()), db0 = uint32_t(dmap.size());
        const size_t ps0 = psmall.size(), us0 = usmall.size(), ds0 = dsmall.size();
        for (uint32_t i = lcount[l]; i < lcount[l + 1]; ++i) {
            const uint32_t q = order[i];
            const uint32_t w = first[q + 1] - first[q], last = first[q + 1] - 1;
            const uint64_t m = nl(last), nt = nu(last);
            meta[i] = make_uint4(first[q], w, uint32_t(m), uint32_t(nt));
            const uint64_t tiles = ((m + UT - 1) / UT) * ((nt + UT - 1) / UT);
            const uint64_t pb = (m + PT - 1) / PT + (w >= 2 ? (nt + TW - 1) / TW : 0);
            if (tiles) ++updating;
            // diagonal blocks: a warp each up to kSnSmallWidth (eight to a block), else a block
            if (w > kSnSmallWidth)
                dmap.push_back(make_uint2(i, 0u));
            else if (w >= 2)
                dsmall.push_back(i);
            if (pmap.size() + pb > UINT32_MAX || umap.size() + tiles > UINT32_MAX ||
                uint64_t(tgt[i]) + nt > UINT32_MAX)
                return set_error(GLU_ERR_UNSUPPORTED, "supernodal schedule too large");
            // small supernodes: one warp each, grouped four (panel) or eight (update) to a block
            const bool small = h->tune.sn_small && w <= kSnSmallWidth && m <= 32 && nt <= 32;
            if (pb && small)
                psmall.push_back(i);
            else if (pb) {
                for (uint64_t bb = 0; bb < pb; ++bb) pmap.push_back(make_uint2(i, uint32_t(bb)));
                panel_w = std::max(panel_w, w);
            }
            // rows [row_cut, m) x targets [tgt_cut, nt): the deferred corner
            const uint64_t row_cut = deferred[q] ? m - ca[q] : m, tgt_cut = deferred[q] ? nt - cb[q] : nt;
            cut[i] = make_uint2(uint32_t(row_cut), uint32_t(tgt_cut));
            const uint64_t nrt = (m + UT - 1) / UT;
            if (tiles && small && m * nt <= 256)
                usmall.push_back(i);
            else
                for (uint64_t bb = 0; bb < tiles; ++bb)
                    if ((bb % nrt) * UT < row_cut || (bb / nrt) * UT < tgt_cut)
                        umap.push_back(make_uint2(i, uint32_t(bb)));
            tgt[i + 1] = tgt[i] + uint32_t(nt);
            pos_off[i + 1] = pos_off[i] + m * nt;
            const double kept = double(m) * nt - double(m - row_cut) * (nt - tgt_cut);
            upd_flops += 2.0 * kept * w;
            upd_bytes += 4.0 * (double(m) * w + double(w) * nt) + 8.0 * kept;
            pan_bytes += 8.0 * (double(m) * w + double(w) * nt) + (w >= 2 ? 8.0 * w * w : 0.0);
        }
        for (size_t g = ps0; g < psmall.size(); g += kSnPanelThreads / 32)
            pmap.push_back(make_uint2(uint32_t(g), kSnSmallFlag | uint32_t(std::min<size_t>(kSnPanelThreads / 32,
                                                                                             psmall.size() - g))));
        for (size_t g = us0; g < usmall.size(); g += 8)
            umap.push_back(make_uint2(uint32_t(g), kSnSmallFlag | uint32_t(std::min<size_t>(8, usmall.size() - g))));
        for (size_t g = ds0; g < dsmall.size(); g += kSnDiagSmallPerBlock)
            dmap.push_back(make_uint2(uint32_t(g), kSnSmallFlag | uint32_t(std::min<size_t>(kSnDiagSmallPerBlock,
                                                                                             dsmall.size() - g))));
        const uint32_t i0 = lcount[l], i1 = lcount[l + 1];
        h->sn_levels.push_back(SnLevel{i0, i1, pb0, uint32_t(pmap.size()) - pb0, ub0, uint32_t(umap.size()) - ub0,
                                       db0, uint32_t(dmap.size()) - db0, updating > 1 ? 1u : 0u, panel_w});
    }
    h->nsn = ns;
    GLU_CUDA(upload(h->d_sn_meta, meta), "upload supernodes");
    GLU_CUDA(upload(h->d_sn_dmap, dmap), "upload supernodes");
    GLU_CUDA(upload(h->d_sn_dsmall, dsmall), "upload supernodes");
    GLU_CUDA(upload(h->d_sn_pmap, pmap), "upload supernodes");
    GLU_CUDA(upload(h->d_sn_umap, umap), "upload supernodes");
    GLU_CUDA(upload(h->d_sn_psmall, psmall), "upload supernodes");
    GLU_CUDA(upload(h->d_sn_usmall, usmall), "upload supernodes");
    GLU_CUDA(upload(h->d_sn_tgt_off, tgt), "upload supernodes");
    GLU_CUDA(upload(h->d_sn_pos_off, pos_off), "upload supernodes");
    if (h->couple_cols) GLU_CUDA(upload(h->d_sn_cut, cut), "upload coupling plan");
    GLU_CUDA(h->d_sn_tgt.alloc(sizeof(uint4) * std::max<uint32_t>(tgt[ns], 1)), "allocate supernode targets");
    h->SN = SnPlanDev{h->d_sn_meta.as<uint4>(),      h->d_sn_dmap.as<uint2>(),  h->d_sn_dsmall.as<uint32_t>(),
                      h->d_sn_pmap.as<uint2>(),      h->d_sn_umap.as<uint2>(),
                      h->d_sn_psmall.as<uint32_t>(), h->d_sn_usmall.as<uint32_t>(), h->d_sn_tgt_off.as<uint32_t>(),
                      h->d_sn_tgt.as<uint4>(),       nullptr,                    h->d_sn_pos_off.as<uint64_t>()};
    if (h->couple_cols) h->SN.cut = h->d_sn_cut.as<uint2>();
    GLU_CUDA(launch_sn_targets(h->P, h->SN, ns, h->d_sn_tgt.as<uint4>(), 0), "supernode targets");
    GLU_CUDA(cudaDeviceSynchronize(), "supernode targets");
    // Position table of the update scatter, when it fits in a quarter of the
    // free memory (the values of every value set are allocated by now) and
    // the tables of all handles on the device stay within a quarter of its
    // memory (many handles on one GPU must not each claim a quarter of what
    // is left).  Without it an update entry in a complete in-place dense tail
    // computes its position, any other searches its target column's rows.
    h->d_sn_pos.release();
    if (h->pos_bytes && h->device < kMaxDevices) g_pos_bytes[h->device] -= h->pos_bytes;
    h->pos_bytes = 0;
    const uint64_t entries = pos_off[ns];
    const uint64_t table_bytes = sizeof(uint32_t) * entries;
    size_t free_b = 0, total_b = 0;
    if (entries > 0 && h->device < kMaxDevices && cudaMemGetInfo(&free_b, &total_b) == cudaSuccess &&
        double(table_bytes) <= 0.25 * double(free_b) &&
        double(g_pos_bytes[h->device].load() + table_bytes) <= 0.25 * double(total_b) &&
        h->d_sn_pos.alloc(table_bytes) == cudaSuccess) {
        g_pos_bytes[h->device] += table_bytes;
        h->pos_bytes = table_bytes;
        GLU_CUDA(launch_sn_positions(h->P, h->SN, ns, h->d_sn_pos.as<uint32_t>(), 0), "supernode positions");
        GLU_CUDA(cudaDeviceSynchronize(), "supernode positions");
        h->SN.pos = h->d_sn_pos.as<uint32_t>();
        upd_bytes += 4.0 * double(entries);
    }
    cudaGetLastError();
    // supernodal solve sweeps: L forward (waits for the supernodes whose L21
    // rows fall in it), U backward (waits for the supernodes holding its targets)
    for (int u = 0; u < 2; ++u) {
        std::vector<int32_t> sl(ns, 0);
        int32_t snl = 0;
        for (uint32_t qq = 0; qq < ns; ++qq) {
            const uint32_t q = u ? ns - 1 - qq : qq;
            const uint32_t s0 = first[q], last = first[q + 1] - 1;
            int32_t mx = -1;
            if (!u) {
                for (uint32_t c = s0; c <= last; ++c)
                    for (uint32_t e = s.csr_r_ptr[c]; e < s.csr_diag_ptr[c]; ++e) {
                        const uint32_t c2 = s.csr_c_idx[e];
                        if (c2 < s0) mx = std::max(mx, sl[sn_of[c2]]);
                    }
            } else {
                for (uint32_t e = s.csr_diag_ptr[last] + 1; e < s.csr_r_ptr[last + 1]; ++e) {
                    const uint32_t j = s.csr_c_idx[e];
                    if (j < t) mx = std::max(mx, sl[sn_of[j]]);
                }
            }
            sl[q] = mx + 1;
            snl = std::max(snl, mx + 2);
        }
        std::vector<uint32_t> lc(size_t(snl) + 1, 0);
        for (uint32_t q = 0; q < ns; ++q) lc[sl[q] + 1]++;
        for (int32_t l = 0; l < snl; ++l) lc[l + 1] += lc[l];
        std::vector<uint32_t> ord(ns);
        {
            std::vector<uint32_t> cur(lc.begin(), lc.end() - 1);
            for (uint32_t q = 0; q < ns; ++q) ord[cur[sl[q]]++] = q;
        }
        std::vector<uint4> smeta(ns);
        std::vector<uint2> smap;
        std::vector<uint32_t> ssmall;
        h->ss_levels[u].clear();
        for (int32_t l = 0; l < snl; ++l) {
            const uint32_t b0 = uint32_t(smap.size());
            const size_t small0 = ssmall.size();
            for (uint32_t i = lc[l]; i < lc[l + 1]; ++i) {
                const uint32_t q = ord[i];
                const uint32_t s0 = first[q], w = first[q + 1] - s0, last = first[q + 1] - 1;
                uint64_t work, off;
                if (!u) {
                    smeta[i] = make_uint4(s0, w, s.l_col_ptr[last] + 1, nl(last));
                    off = nl(last);
                    work = (off + kSnSweepRows - 1) / kSnSweepRows;
                } else {
                    off = 0;
                    for (uint32_t c = s0; c <= last; ++c) off += (s.l_col_ptr[c] - (c - s0)) - s.sym_c_ptr[c];
                    smeta[i] = make_uint4(s0, w, 0u, 0u);
                    work = (off + kSnSweepAbove - 1) / kSnSweepAbove;
                }
                if (h->tune.sn_small && w <= kSnSmallWidth && off <= 32) {
                    ssmall.push_back(i);
                    continue;
                }
                work = std::max<uint64_t>(work, 1);
                if (smap.size() + work > UINT32_MAX) return set_error(GLU_ERR_UNSUPPORTED, "solve schedule too large");
                for (uint64_t bb = 0; bb < work; ++bb) smap.push_back(make_uint2(i, uint32_t(bb)));
            }
            const uint32_t big = uint32_t(smap.size()) - b0;
            for (size_t g = small0; g < ssmall.size(); g += 8)
                smap.push_back(make_uint2(uint32_t(g), kSnSmallFlag | uint32_t(std::min<size_t>(8, ssmall.size() - g))));
            h->ss_levels[u].push_back(SnSweepLevel{b0, uint32_t(smap.size()) - b0, big});
        }
        // fused form: per block the supernodes it solves (waits for) and the
        // supernodes whose unknowns its scatter updates (releases)
        std::vector<uint32_t> pos_of(ns);  // supernode -> sweep-order index
        for (uint32_t i = 0; i < ns; ++i) pos_of[ord[i]] = i;
        std::vector<uint32_t> woff(1, 0), widx, roff(1, 0), ridx, indeg(ns, 0), mark(ns, UINT32_MAX);
        auto release_rows = [&](uint32_t blk, uint32_t p0, uint32_t p1, bool by_csc_row) {
            // targets of the entries [p0, p1): rows of column entries (CSC)
            for (uint32_t p = p0; p < p1; ++p) {
                const uint32_t r = s.sym_r_idx[p];
                (void)by_csc_row;
                if (r >= t) continue;  // tail rows: solved by a later launch
                const uint32_t q = pos_of[sn_of[r]];
                if (mark[q] != blk) {
                    mark[q] = blk;
                    ridx.push_back(q);
                    ++indeg[q];
                }
            }
        };
        for (uint32_t blk = 0; blk < uint32_t(smap.size()); ++blk) {
            const uint2 bi = smap[blk];
            std::vector<uint32_t> mine;
            if (bi.y & kSnSmallFlag) {
                for (uint32_t g = 0; g < (bi.y & ~kSnSmallFlag); ++g) mine.push_back(ssmall[bi.x + g]);
            } else {
                mine.push_back(bi.x);
            }
            for (uint32_t i : mine) widx.push_back(i);
            woff.push_back(uint32_t(widx.size()));
            for (uint32_t i : mine) {
                const uint32_t q = ord[i];
                const uint32_t s0 = first[q], w = first[q + 1] - s0, last = first[q + 1] - 1;
                const bool part_all = bi.y & kSnSmallFlag;
                if (!u) {
                    // L21 rows of this block: all (small) or the block's chunk of kSnSweepRows
                    const uint32_t lb = s.l_col_ptr[last] + 1, m = nl(last);
                    const uint32_t r0 = part_all ? 0 : bi.y * kSnSweepRows, r1 = part_all ? m : std::min(m, r0 + kSnSweepRows);
                    release_rows(blk, lb + r0, lb + r1, true);
                } else {
                    // entries above the block in the supernode's columns, in column order
                    uint32_t e = 0;
                    const uint32_t e0 = part_all ? 0 : bi.y * kSnSweepAbove, e1 = part_all ? UINT32_MAX : e0 + kSnSweepAbove;
                    for (uint32_t c = s0; c <= last; ++c) {
                        const uint32_t p0 = s.sym_c_ptr[c], p1 = s.l_col_ptr[c] - (c - s0);
                        const uint32_t cnt = p1 - p0;
                        const uint32_t lo = std::max(e, e0), hi = std::min(e + cnt, e1);
                        if (lo < hi) release_rows(blk, p0 + (lo - e), p0 + (hi - e), true);
                        e += cnt;
                    }
                    (void)w;
                }
            }
            roff.push_back(uint32_t(ridx.size()));
        }
        GLU_CUDA(upload(h->d_ss_woff[u], woff), "upload solve plan");
        GLU_CUDA(upload(h->d_ss_widx[u], widx), "upload solve plan");
        GLU_CUDA(upload(h->d_ss_roff[u], roff), "upload solve plan");
        GLU_CUDA(upload(h->d_ss_ridx[u], ridx), "upload solve plan");
        GLU_CUDA(upload(h->d_ss_indeg[u], indeg), "upload solve plan");
        GLU_CUDA(upload(h->d_ss_small[u], ssmall), "upload solve plan");
        GLU_CUDA(upload(h->d_ss_map[u], smap), "upload solve plan");
        GLU_CUDA(upload(h->d_ss_meta[u], smeta), "upload solve plan");
        SnSweepPlan &pl = h->S.sn[u];
        pl.map = h->d_ss_map[u].as<uint2>();
        pl.meta = h->d_ss_meta[u].as<uint4>();
        pl.small = h->d_ss_small[u].as<uint32_t>();
        pl.levels = h->ss_levels[u].data();
        pl.nlev = uint32_t(h->ss_levels[u].size());
        pl.fused = h->tune.sn_sweep_fused;
        pl.nblocks = uint32_t(smap.size());
        pl.ns = ns;
        pl.wait_off = h->d_ss_woff[u].as<uint32_t>();
        pl.wait_idx = h->d_ss_widx[u].as<uint32_t>();
        pl.rel_off = h->d_ss_roff[u].as<uint32_t>();
        pl.rel_idx = h->d_ss_ridx[u].as<uint32_t>();
        pl.indeg = h->d_ss_indeg[u].as<uint32_t>();
        h->stats.sn_sweep_levels += pl.nlev;
    }
    h->stats.sn_update_flops = upd_flops;
    h->stats.sn_update_bytes = upd_bytes;
    h->stats.sn_panel_bytes = pan_bytes;
    return GLU_OK;
}

Status build_plan(glu_handle_s *h) {
    const SymbolicData &s = h->pat;
    const uint32_t n = h->n;
    // split point: fully dense trailing block (factored in place) or, when the
    // cost model prefers a larger block, a dense buffer of order <= max_m
    uint32_t t_full, m_full;
    find_full_tail(s, 1, t_full, m_full);
    uint32_t max_m = h->tune.dense_tail_max;
    {
        // buffers for every value set must fit in a fraction of free memory
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && free_b > 0) {
            double cap = std::sqrt(0.4 * double(free_b) / (4.0 * h->batch));
            if (cap < max_m) max_m = uint32_t(cap);
        }
    }
    uint32_t t_opt = choose_split(s, h->level_ptr, h->level_idx, std::max(max_m, m_full), h->tune);
    h->dense_buffer = false;
    if (t_opt >= t_full) {
        h->t = t_opt;  // any trailing block of a fully dense block is fully dense
    } else if (n - t_opt <= max_m) {
        h->t = t_opt;
        h->dense_buffer = true;
    } else {
        h->t = t_full;
    }
    h->m = n - h->t;
    if (h->m < h->tune.dense_tail_min) {
        h->t = n;
        h->m = 0;
        h->dense_buffer = false;
    }
    const uint32_t t = h->t, m = h->m;
    h->doff_h.assign(std::max<uint32_t>(m, 1), 0);
    h->tail_start_h.assign(std::max<uint32_t>(m, 1), 0);
    for (uint32_t j = 0; j < m; ++j) {
        const uint32_t *b0 = s.sym_r_idx.data() + s.sym_c_ptr[t + j];
        const uint32_t *b1 = s.sym_r_idx.data() + s.sym_c_ptr[t + j + 1];
        h->tail_start_h[j] = uint32_t(std::lower_bound(b0, b1, t) - s.sym_r_idx.data());
        h->doff_h[j] = h->dense_buffer ? j * m : h->tail_start_h[j];
    }
    h->d_dense.release();
    if (h->dense_buffer)
        GLU_CUDA(h->d_dense.alloc(sizeof(float) * size_t(m) * m * h->batch), "allocate dense tail buffer");
    GLU_CUDA(upload(h->d_tail_start, h->tail_start_h), "upload dense offsets");

    std::vector<uint32_t> sched, item_off(1, 0);
    h->levels_h.clear();
    h->items_h.clear();
    h->work_h.clear();
    double flops = 0;
    for (uint32_t k = 0; k < n; ++k) {
        double L = s.sym_c_ptr[k + 1] - s.l_col_ptr[k] - 1;
        double U = s.csr_r_ptr[k + 1] - s.csr_diag_ptr[k] - 1;
        flops += L + 2 * L * U;
    }
    h->flops = flops;
    for (int32_t l = 0; l < h->num_lev; ++l) {
        uint32_t s0 = uint32_t(sched.size());
        double sumL = 0;
        uint32_t cols = 0;
        for (int32_t q = h->level_ptr[l]; q < h->level_ptr[l + 1]; ++q) {
            uint32_t k = uint32_t(h->level_idx[q]);
            if (k >= t) break;  // ascending within a level
            uint32_t L = s.sym_c_ptr[k + 1] - s.l_col_ptr[k] - 1;
            if (L == 0) continue;
            sched.push_back(k);
            sumL += L;
            ++cols;
        }
        if (cols == 0) continue;
        uint32_t G = pick_group(sumL / cols, h->tune.group_lanes);
        uint32_t CH = G * kItemUnroll;
        uint32_t s1 = uint32_t(sched.size());
        uint64_t items = 0, work = 0;
        uint32_t active = 0;
        for (uint32_t q = s0; q < s1; ++q) {
            uint32_t k = sched[q];
            uint64_t L = s.sym_c_ptr[k + 1] - s.l_col_ptr[k] - 1;
            uint64_t U = s.csr_r_ptr[k + 1] - s.csr_diag_ptr[k] - 1;
            uint64_t it = U * ((L + CH - 1) / CH);
            items += it;
            work += L * U;
            if (it) ++active;
            uint64_t next = uint64_t(item_off.back()) + it;
            if (next > UINT32_MAX) return set_error(GLU_ERR_UNSUPPORTED, "too many work items");
            item_off.push_back(uint32_t(next));
        }
        h->levels_h.push_back(LevelInfo{s0, s1, G, active > 1 ? 1u : 0u});
        h->items_h.push_back(uint32_t(items));
        h->work_h.push_back(work);
    }
    // steps: narrow runs go to the cluster kernel
    h->steps.clear();
    const uint32_t NL = uint32_t(h->levels_h.size());
    uint32_t l = 0;
    while (l < NL) {
        if (h->work_h[l] > h->tune.wide_work || h->tune.chain_cluster == 0) {
            h->steps.push_back(Step{STEP_LEVEL, l, l + 1});
            ++l;
        } else {
            uint32_t e = l;
            while (e < NL && h->work_h[e] <= h->tune.wide_work) ++e;
            if (e - l == 1)
                h->steps.push_back(Step{STEP_LEVEL, l, e});
            else
                h->steps.push_back(Step{STEP_CHAIN, l, e});
            l = e;
        }
    }
    GLU_CUDA(upload(h->d_sched, sched), "upload schedule");
    GLU_CUDA(upload(h->d_item_off, item_off), "upload schedule");
    GLU_CUDA(upload(h->d_levels, h->levels_h), "upload schedule");
    GLU_CUDA(upload(h->d_doff, h->doff_h), "upload dense offsets");
    h->F.sched_cols = h->d_sched.as<uint32_t>();
    h->F.item_off = h->d_item_off.as<uint32_t>();
    h->F.levels = h->d_levels.as<LevelInfo>();

    // solve plan: level schedules of the four sparse sweeps
    h->S.t = t;
    h->S.m = m;
    h->S.doff = h->d_doff.as<uint32_t>();
    h->S.tail_start = h->d_tail_start.as<uint32_t>();
    h->S.cluster = h->tune.solve_cluster ? h->tune.solve_cluster : 4;
    h->S.spin_limit = h->spin_limit;
    h->S.ticket_base = 0;
    {
        // CSR position of the first column >= t in every tail row
        std::vector<uint32_t> trs(std::max<uint32_t>(m, 1), 0);
        for (uint32_t i = 0; i < m; ++i) {
            const uint32_t *b0 = s.csr_c_idx.data() + s.csr_r_ptr[t + i];
            const uint32_t *b1 = s.csr_c_idx.data() + s.csr_r_ptr[t + i + 1];
            trs[i] = uint32_t(std::lower_bound(b0, b1, t) - s.csr_c_idx.data());
        }
        GLU_CUDA(upload(h->d_tail_row_start, trs), "upload solve plan");
        h->S.tail_row_start = h->d_tail_row_start.as<uint32_t>();
    }
    for (int mode = 0; mode < 4; ++mode) {
        std::vector<uint32_t> cols, lptr, ioff;
        build_sweep(s, t, mode, h->tune.solve_thin, cols, lptr, ioff, h->sw_steps[mode]);
        GLU_CUDA(upload(h->d_sw_cols[mode], cols), "upload solve plan");
        GLU_CUDA(upload(h->d_sw_lptr[mode], lptr), "upload solve plan");
        GLU_CUDA(upload(h->d_sw_ioff[mode], ioff), "upload solve plan");
        SweepPlan &sp = h->S.sweep[mode];
        sp.cols = h->d_sw_cols[mode].as<uint32_t>();
        sp.lptr = h->d_sw_lptr[mode].as<uint32_t>();
        sp.item_off = h->d_sw_ioff[mode].as<uint32_t>();
        sp.steps = h->sw_steps[mode].data();
        sp.nsteps = uint32_t(h->sw_steps[mode].size());
        sp.nlev = uint32_t(lptr.size() - 1);
    }

    Status sn = build_sn_plan(h);
    if (sn != GLU_OK) return sn;
    h->SN.tail_start = h->d_tail_start.as<uint32_t>();
    h->SN.t = t;
    h->SN.tail_full = (m > 0 && !h->dense_buffer) ? 1u : 0u;
    uint32_t wide = 0, chains = 0;
    for (auto &st : h->steps) (st.kind == STEP_CHAIN ? chains : wide)++;
    h->stats.wide_levels = h->use_sn ? 0 : wide;
    h->stats.chain_segments = h->use_sn ? 0 : chains;
    h->stats.dense_tail = m;
    h->stats.factor_flops = flops;
    h->stats.supernodes = h->nsn;
    h->stats.couple_columns = h->couple_cols;
    h->stats.couple_groups = uint32_t(h->couple_groups.size());
    h->stats.sn_levels = uint32_t(h->sn_levels.size());
    uint64_t launches = 2;
    if (h->use_sn) {
        for (const SnLevel &lv : h->sn_levels) launches += (lv.dblocks ? 1 : 0) + (lv.pblocks ? 1 : 0) + (lv.ublocks ? 1 : 0);
    } else {
        launches += h->steps.size() + (NL ? 1 : 0);
    }
    if (m) launches += 2 * ((m + kDenseNB - 1) / kDenseNB) + (h->dense_buffer ? 2 : 0) + 2 * h->couple_groups.size();
    h->stats.factor_launches = launches;
    return GLU_OK;
}

Status identity_transform(glu_handle_s *h) {
    std::vector<uint32_t> id(h->n);
    std::iota(id.begin(), id.end(), 0u);
    for (int k = 0; k < 4; ++k) {
        GLU_CUDA(upload(h->d_tr[2 * k], id), "upload transform");
        h->d_tr[2 * k + 1].release();
    }
    h->T = TransformDev{h->d_tr[0].as<uint32_t>(), nullptr, h->d_tr[2].as<uint32_t>(), nullptr,
                        h->d_tr[4].as<uint32_t>(), nullptr, h->d_tr[6].as<uint32_t>(), nullptr};
    return GLU_OK;
}

Status create_handle(int device, SymbolicData &&s, uint32_t batch, glu_handle_t *out) {
    if (!out) return set_error(GLU_ERR_ARG, "null output handle");
    *out = nullptr;
    if (batch == 0) return set_error(GLU_ERR_ARG, "batch must be positive");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return set_error(GLU_ERR_NO_DEVICE, "no CUDA device available");
    if (device < 0 || device >= ndev) return set_error(GLU_ERR_ARG, "device %d out of range", device);
    DeviceGuard g(device);
    std::unique_ptr<glu_handle_s> h(new glu_handle_s());
    h->device = device;
    h->n = s.n;
    h->nnz = s.nnz;
    h->batch = batch;
    h->pat = std::move(s);
    h->tune = glu_tuning{200000u, 16u, 0u, 64u, 4096u, 128u, 4u, kSnMaxWidth, 1u, kLookaheadMin, kDenseTcMin, 0u, 0u,
                         0u, 1u, kDenseGroupMax};
    const SymbolicData &p = h->pat;
    GLU_CUDA(upload(h->d_cptr, p.sym_c_ptr), "upload pattern");
    GLU_CUDA(upload(h->d_ridx, p.sym_r_idx), "upload pattern");
    GLU_CUDA(upload(h->d_diag, p.l_col_ptr), "upload pattern");
    GLU_CUDA(upload(h->d_rptr, p.csr_r_ptr), "upload pattern");
    GLU_CUDA(upload(h->d_cidx, p.csr_c_idx), "upload pattern");
    GLU_CUDA(upload(h->d_rdiag, p.csr_diag_ptr), "upload pattern");
    GLU_CUDA(upload(h->d_cpos, p.csr_pos), "upload pattern");
    h->P = DevPattern{h->d_cptr.as<uint32_t>(), h->d_ridx.as<uint32_t>(), h->d_diag.as<uint32_t>(),
                      h->d_rptr.as<uint32_t>(), h->d_cidx.as<uint32_t>(), h->d_rdiag.as<uint32_t>(),
                      h->d_cpos.as<uint32_t>(), h->n, h->nnz};
    GLU_CUDA(h->d_val.alloc(sizeof(float) * size_t(h->nnz) * batch), "allocate values");
    GLU_CUDA(cudaMemset(h->d_val.p, 0, sizeof(float) * size_t(h->nnz) * batch), "clear values");
    GLU_CUDA(h->d_status.alloc(256), "allocate status");
    GLU_CUDA(cudaMemset(h->d_status.p, 0, 256), "clear status");
    GLU_CUDA(h->d_pert.alloc(sizeof(float) * batch), "allocate");
    GLU_CUDA(h->d_colmax.alloc(sizeof(float) * batch), "allocate");
    GLU_CUDA(h->d_diag_scratch.alloc(sizeof(float) * kDenseNB * kDenseNB * batch), "allocate");
    GLU_CUDA(h->d_counters.alloc(sizeof(uint32_t) * (size_t(h->n) + 64)), "allocate");
    GLU_CUDA(h->d_ticket.alloc(256), "allocate");
    GLU_CUDA(cudaMallocHost(reinterpret_cast<void **>(&h->h_status), 256), "allocate pinned");
    GLU_CUDA(cudaEventCreate(&h->ev0), "event");
    GLU_CUDA(cudaEventCreate(&h->ev1), "event");
    {
        int sms = 0;
        GLU_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "device attribute");
        h->num_sms = uint32_t(std::max(sms, 1));
    }
    {
        int least = 0, greatest = 0;
        GLU_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest), "stream priorities");
        GLU_CUDA(cudaStreamCreateWithPriority(&h->aux, cudaStreamNonBlocking, greatest), "stream");
    }
    GLU_CUDA(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming), "event");
    GLU_CUDA(cudaEventCreateWithFlags(&h->ev_panel, cudaEventDisableTiming), "event");
    GLU_CUDA(cudaEventCreateWithFlags(&h->ev_rest, cudaEventDisableTiming), "event");

    // level sets on the device
    {
        DevBuf scratch, level_of, lptr, lidx, nlev;
        GLU_CUDA(scratch.alloc(level_scratch_bytes(h->n)), "allocate level scratch");
        GLU_CUDA(level_of.alloc(sizeof(int32_t) * h->n), "allocate levels");
        GLU_CUDA(lptr.alloc(sizeof(int32_t) * (size_t(h->n) + 1)), "allocate levels");
        GLU_CUDA(lidx.alloc(sizeof(int32_t) * h->n), "allocate levels");
        GLU_CUDA(nlev.alloc(sizeof(int32_t)), "allocate levels");
        GLU_CUDA(build_levels(h->P, scratch.p, level_of.as<int32_t>(), lptr.as<int32_t>(),
                              lidx.as<int32_t>(), nlev.as<int32_t>(), h->d_status.as<uint32_t>(), 0),
                 "build levels");
        GLU_CUDA(cudaMemcpy(&h->num_lev, nlev.p, sizeof(int32_t), cudaMemcpyDeviceToHost), "levels");
        uint32_t st = 0;
        GLU_CUDA(cudaMemcpy(&st, h->d_status.p, sizeof(uint32_t), cudaMemcpyDeviceToHost), "levels");
        if (st & DEV_TIMEOUT) return set_error(GLU_ERR_TIMEOUT, "level construction wait timed out");
        h->level_ptr.resize(size_t(h->num_lev) + 1);
        h->level_idx.resize(h->n);
        GLU_CUDA(cudaMemcpy(h->level_ptr.data(), lptr.p, sizeof(int32_t) * h->level_ptr.size(),
                            cudaMemcpyDeviceToHost), "levels");
        GLU_CUDA(cudaMemcpy(h->level_idx.data(), lidx.p, sizeof(int32_t) * h->n, cudaMemcpyDeviceToHost),
                 "levels");
    }
    int maxc = 0;
    h->chain_cluster = 16;
    {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(16, 1, 1);
        cfg.blockDim = dim3(kChainThreads, 1, 1);
        cudaLaunchAttribute a[1];
        a[0].id = cudaLaunchAttributeClusterDimension;
        a[0].val.clusterDim.x = 16;
        a[0].val.clusterDim.y = 1;
        a[0].val.clusterDim.z = 1;
        cfg.attrs = a;
        cfg.numAttrs = 1;
        cudaFuncSetAttribute(chain_kernel_ptr(), cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (cudaOccupancyMaxActiveClusters(&maxc, chain_kernel_ptr(), &cfg) != cudaSuccess || maxc < 1)
            h->chain_cluster = 8;
        cudaGetLastError();
    }
    h->tune.chain_cluster = h->chain_cluster;
    Status st = build_plan(h.get());
    if (st != GLU_OK) return st;
    st = identity_transform(h.get());
    if (st != GLU_OK) return st;
    h->stats.n = h->n;
    h->stats.nnz_lu = h->nnz;
    h->stats.batch = batch;
    h->stats.num_lev = h->num_lev;
    *out = h.release();
    return GLU_OK;
}

Status check_range(glu_handle_s *h, uint32_t first, uint32_t count) {
    if (count == 0 || first >= h->batch || count > h->batch - first)
        return set_error(GLU_ERR_ARG, "value sets [%u, %u) outside batch %u", first, first + count, h->batch);
    return GLU_OK;
}

Status read_status(glu_handle_s *h, cudaStream_t st, uint32_t *flags) {
    GLU_CUDA(cudaMemcpyAsync(h->h_status, h->d_status.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, st),
             "read status");
    GLU_CUDA(cudaStreamSynchronize(st), "synchronize");
    *flags = h->h_status[0];
    return GLU_OK;
}

// Kernels one FP32 solve (both triangular sweeps) launches, from the plan.
uint64_t solve_kernel_count(const glu_handle_s *h, bool trans) {
    uint64_t k = 0;
    const SolvePlanDev &S = h->S;
    for (int u = 0; u < 2; ++u) {
        const bool sn = !trans && S.sn[u].nlev;
        if (sn) {
            uint32_t lev = 0;
            for (uint32_t l = 0; l < S.sn[u].nlev; ++l) {
                const uint2 k2 = sn_sweep_level_launches(S.sn[u].levels[l], u == 1);
                lev += k2.x + k2.y;
            }
            k += (S.sn[u].fused && h->use_sn ? 1 : lev) + (S.t > 0 ? 1 : 0);
        } else {
            const int mode = trans ? (u == 0 ? SWEEP_UT : SWEEP_LT) : (u == 0 ? SWEEP_L : SWEEP_U);
            k += S.sweep[mode].nsteps + ((mode == SWEEP_U || mode == SWEEP_UT) && S.t > 0 ? 1 : 0);
        }
    }
    if (S.m) k += 2 + (S.t > 0 ? 1 : 0);  // two dense sweeps, the tail coupling
    return k;
}

// Floats of the dense tail's diagonal-block inverses of one value set.
size_t dinv_per_set(const glu_handle_s *h) { return size_t((h->m + 63) / 64) * 2 * 64 * 64; }

// The solve plan of the next solve: the handle's, with a pending
// GLU_INJECT_UNSET_SOLVE_FLAG applied (and consumed).
SolvePlanDev solve_plan(glu_handle_s *h) {
    SolvePlanDev S = h->S;
    if (h->inject_unset_flag) {
        S.ticket_base = 1;
        h->inject_unset_flag = false;
    }
    return S;
}

// One FP32 solve of y in place (nrhs vectors of n per value set), in the
// permuted system, with the factors of value sets [z, z + count).
Status solve_inplace(glu_handle_s *h, uint32_t z, uint32_t count, float *y, uint32_t nrhs, bool trans,
                     cudaStream_t st) {
    const uint32_t nb = (h->m + 63) / 64 + 1;
    GLU_CUDA(h->d_flags.ensure(sizeof(uint32_t) * size_t(nb) * count), "allocate solve flags");
    GLU_CUDA(h->d_ticket.ensure(sizeof(uint32_t) * std::max<size_t>(count, 64)), "allocate solve flags");
    uint32_t *cnt = h->d_flags.as<uint32_t>();
    uint32_t *tk = h->d_ticket.as<uint32_t>();
    uint32_t *status = h->d_status.as<uint32_t>();
    const float *val = h->d_val.as<float>() + size_t(z) * h->nnz;
    const float *dval = h->dense_buffer ? h->d_dense.as<float>() + size_t(z) * h->m * h->m : val;
    SolveBatch B;
    B.count = count;
    B.vstride = h->nnz;
    B.dstride = h->dense_buffer ? uint64_t(h->m) * h->m : h->nnz;
    B.dinv = h->m ? h->d_dinv.as<float>() + size_t(z) * dinv_per_set(h) : nullptr;
    if (h->tune.sn_sweep_fused && h->use_sn) {
        const size_t ns = std::max(h->S.sn[0].ns, h->S.sn[1].ns);
        GLU_CUDA(h->d_sweep_done.ensure(sizeof(uint32_t) * ns * count + 4), "allocate sweep counters");
        B.sweep_done = h->d_sweep_done.as<uint32_t>();
    }
    GLU_CUDA(h->d_xo.ensure(sizeof(float) * size_t(h->n) * nrhs * count), "allocate solve buffer");
    float *xo = h->d_xo.as<float>();
    const SolvePlanDev S = solve_plan(h);
    h->stats.solve_launches += solve_kernel_count(h, trans);
    if (!trans) {
        GLU_CUDA(solve_lower_unit(h->P, S, val, dval, y, xo, nrhs, cnt, tk, status, B, st), "lower solve");
        GLU_CUDA(solve_upper(h->P, S, val, dval, y, xo, nrhs, cnt, tk, status, B, st), "upper solve");
    } else {
        GLU_CUDA(solve_upper_trans(h->P, S, val, dval, y, xo, nrhs, cnt, tk, status, B, st),
                 "transposed upper solve");
        GLU_CUDA(solve_lower_unit_trans(h->P, S, val, dval, y, xo, nrhs, cnt, tk, status, B, st),
                 "transposed lower solve");
    }
    return GLU_OK;
}

Status solve_f32(glu_handle_s *h, uint32_t inst, uint32_t nrhs, const float *b, float *x,
                 glu_memory where, bool trans, cudaStream_t st) {
    if (!h->factored) return set_error(GLU_ERR_STATE, "solve before factorization");
    if (inst >= h->batch) return set_error(GLU_ERR_ARG, "value set %u outside batch", inst);
    if (nrhs == 0) return GLU_OK;
    if (!b || !x) return set_error(GLU_ERR_ARG, "null vector");
    DeviceGuard g(h->device);
    const size_t len = size_t(h->n) * nrhs;
    GLU_CUDA(h->d_y.ensure(sizeof(float) * len), "allocate solve buffer");
    GLU_CUDA(h->d_io32.ensure(sizeof(float) * len), "allocate solve buffer");
    float *y = h->d_y.as<float>();
    float *io = h->d_io32.as<float>();
    const float *bin = b;
    if (where == GLU_HOST) {
        GLU_CUDA(cudaMemcpyAsync(io, b, sizeof(float) * len, cudaMemcpyHostToDevice, st), "copy b");
        bin = io;
    }
    GLU_CUDA(cudaMemsetAsync(h->d_status.p, 0, sizeof(uint32_t), st), "reset status");
    const TransformDev &T = h->T;
    h->stats.solve_launches = 2;  // the two transforms; solve_inplace adds the sweeps
    GLU_CUDA(launch_transform_f32(trans ? T.tin_idx : T.in_idx, trans ? T.tin_scale : T.in_scale, bin, y,
                                  h->n, nrhs, st), "transform");
    Status s = solve_inplace(h, inst, 1, y, nrhs, trans, st);
    if (s != GLU_OK) return s;
    float *xout = (where == GLU_HOST) ? io : x;
    GLU_CUDA(launch_transform_f32(trans ? T.tout_idx : T.out_idx, trans ? T.tout_scale : T.out_scale, y,
                                  xout, h->n, nrhs, st), "transform");
    if (where == GLU_HOST)
        GLU_CUDA(cudaMemcpyAsync(x, io, sizeof(float) * len, cudaMemcpyDeviceToHost, st), "copy x");
    uint32_t flags = 0;
    s = read_status(h, st, &flags);
    if (s != GLU_OK) return s;
    if (flags & DEV_TIMEOUT) return set_error(GLU_ERR_TIMEOUT, "solve dependency wait timed out");
    return GLU_OK;
}

}  // namespace

namespace glu {

int handle_device(const glu_handle_s *h) { return h->device; }

Status solve_f32_scratch(glu_handle_s *h, uint32_t inst, uint32_t nrhs, const float *b, float *x, float *y,
                         float *xo, uint32_t *flags, uint32_t *ticket, size_t max_values, uint32_t max_blocks,
                         void *stream) {
    if (!h->factored) return set_error(GLU_ERR_STATE, "solve before factorization");
    if (inst >= h->batch) return set_error(GLU_ERR_ARG, "value set %u outside batch", inst);
    if (nrhs == 0) return GLU_OK;
    if (!b || !x) return set_error(GLU_ERR_ARG, "null vector");
    if (size_t(h->n) * nrhs > max_values)
        return set_error(GLU_ERR_UNSUPPORTED, "n * nrhs = %zu exceeds the %zu values of the static scratch",
                         size_t(h->n) * nrhs, max_values);
    const uint32_t blocks = (h->m + 63) / 64;
    if (blocks + 1 > max_blocks)
        return set_error(GLU_ERR_UNSUPPORTED, "dense trailing block of order %u exceeds the static scratch", h->m);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    GLU_CUDA(cudaMemsetAsync(h->d_status.p, 0, sizeof(uint32_t), st), "reset status");
    const TransformDev &T = h->T;
    GLU_CUDA(launch_transform_f32(T.in_idx, T.in_scale, b, y, h->n, nrhs, st), "transform");
    const float *val = h->d_val.as<float>() + size_t(inst) * h->nnz;
    const float *dval = h->dense_buffer ? h->d_dense.as<float>() + size_t(inst) * h->m * h->m : val;
    uint32_t *status = h->d_status.as<uint32_t>();
    const SolvePlanDev S = solve_plan(h);
    SolveBatch one;
    one.dinv = h->m ? h->d_dinv.as<float>() + size_t(inst) * dinv_per_set(h) : nullptr;
    GLU_CUDA(solve_lower_unit(h->P, S, val, dval, y, xo, nrhs, flags, ticket, status, one, st), "lower solve");
    GLU_CUDA(solve_upper(h->P, S, val, dval, y, xo, nrhs, flags, ticket, status, one, st), "upper solve");
    GLU_CUDA(launch_transform_f32(T.out_idx, T.out_scale, y, x, h->n, nrhs, st), "transform");
    uint32_t fl = 0;
    Status s = read_status(h, st, &fl);
    if (s != GLU_OK) return s;
    if (fl & DEV_TIMEOUT) return set_error(GLU_ERR_TIMEOUT, "solve dependency wait timed out");
    return GLU_OK;
}

}  // namespace glu

// ===================================================================== C ABI ==
extern "C" {

const char *glu_last_error(void) { return g_last_error.c_str(); }
const char *glu_version(void) { return "glu_b200 0.1 (sm_100a)"; }

glu_status glu_symbolic_analyze(uint32_t n, uint32_t nnz_a, const uint32_t *ap, const uint32_t *ai,
                                glu_symbolic_t *out) {
    if (!out || !ap || (nnz_a && !ai)) return set_error(GLU_ERR_ARG, "null argument");
    *out = nullptr;
    std::unique_ptr<glu_symbolic_s> s(new glu_symbolic_s());
    Status st = symbolic_analyze(n, nnz_a, ap, ai, s->s);
    if (st != GLU_OK) return st;
    *out = s.release();
    return GLU_OK;
}

glu_status glu_symbolic_sizes(glu_symbolic_t s, uint32_t *n, uint32_t *nnz_lu) {
    if (!s) return set_error(GLU_ERR_ARG, "null symbolic handle");
    if (n) *n = s->s.n;
    if (nnz_lu) *nnz_lu = s->s.nnz;
    return GLU_OK;
}

glu_status glu_symbolic_export(glu_symbolic_t s, uint32_t *sym_c_ptr, uint32_t *sym_r_idx,
                               uint32_t *l_col_ptr, uint32_t *csr_r_ptr, uint32_t *csr_c_idx,
                               uint32_t *csr_diag_ptr) {
    if (!s) return set_error(GLU_ERR_ARG, "null symbolic handle");
    const SymbolicData &d = s->s;
    auto cp = [](uint32_t *dst, const std::vector<uint32_t> &v) {
        if (dst && !v.empty()) memcpy(dst, v.data(), sizeof(uint32_t) * v.size());
    };
    cp(sym_c_ptr, d.sym_c_ptr);
    cp(sym_r_idx, d.sym_r_idx);
    cp(l_col_ptr, d.l_col_ptr);
    cp(csr_r_ptr, d.csr_r_ptr);
    cp(csr_c_idx, d.csr_c_idx);
    cp(csr_diag_ptr, d.csr_diag_ptr);
    return GLU_OK;
}

glu_status glu_symbolic_slots(glu_symbolic_t s, uint32_t *a_slot) {
    if (!s || !a_slot) return set_error(GLU_ERR_ARG, "null argument");
    if (!s->s.a_slot.empty()) memcpy(a_slot, s->s.a_slot.data(), sizeof(uint32_t) * s->s.a_slot.size());
    return GLU_OK;
}

glu_status glu_predict_lu(glu_symbolic_t s, const double *ax, float *val) {
    if (!s || !val || (s->s.nnz_a && !ax)) return set_error(GLU_ERR_ARG, "null argument");
    predict_lu(s->s, ax, val);
    return GLU_OK;
}

void glu_symbolic_destroy(glu_symbolic_t s) { delete s; }

glu_status glu_create(glu_symbolic_t s, int device, uint32_t batch, glu_handle_t *out) {
    TraceRange trace_("glu_create");
    if (!s) return set_error(GLU_ERR_ARG, "null symbolic handle");
    SymbolicData copy = s->s;
    return create_handle(device, std::move(copy), batch, out);
}

glu_status glu_create_from_pattern(int device, uint32_t n, uint32_t nnz, const uint32_t *sym_c_ptr,
                                   const uint32_t *sym_r_idx, const uint32_t *l_col_ptr,
                                   const uint32_t *csr_r_ptr, const uint32_t *csr_c_idx,
                                   const uint32_t *csr_diag_ptr, uint32_t batch, glu_handle_t *out) {
    if (!sym_c_ptr || !sym_r_idx || !l_col_ptr || !csr_r_ptr || !csr_c_idx || !csr_diag_ptr)
        return set_error(GLU_ERR_ARG, "null pattern array");
    if (n == 0 || sym_c_ptr[0] != 0 || sym_c_ptr[n] != nnz || csr_r_ptr[0] != 0 || csr_r_ptr[n] != nnz)
        return set_error(GLU_ERR_ARG, "inconsistent pattern");
    // Every pointer array is checked before any array is indexed through it:
    // the planners and the level kernel read the arrays without bounds checks.
    for (uint32_t i = 0; i < n; ++i) {
        if (sym_c_ptr[i] > sym_c_ptr[i + 1]) return set_error(GLU_ERR_ARG, "sym_c_ptr decreases at column %u", i);
        if (csr_r_ptr[i] > csr_r_ptr[i + 1]) return set_error(GLU_ERR_ARG, "csr_r_ptr decreases at row %u", i);
    }
    for (uint32_t i = 0; i < n; ++i) {
        if (csr_diag_ptr[i] < csr_r_ptr[i] || csr_diag_ptr[i] >= csr_r_ptr[i + 1] ||
            csr_c_idx[csr_diag_ptr[i]] != i)
            return set_error(GLU_ERR_ARG, "invalid diagonal pointer of row %u", i);
    }
    SymbolicData s;
    s.n = n;
    s.nnz = nnz;
    s.sym_c_ptr.assign(sym_c_ptr, sym_c_ptr + n + 1);
    s.sym_r_idx.assign(sym_r_idx, sym_r_idx + nnz);
    s.l_col_ptr.assign(l_col_ptr, l_col_ptr + n);
    s.csr_r_ptr.assign(csr_r_ptr, csr_r_ptr + n + 1);
    s.csr_c_idx.assign(csr_c_idx, csr_c_idx + nnz);
    s.csr_diag_ptr.assign(csr_diag_ptr, csr_diag_ptr + n);
    for (uint32_t i = 0; i < n; ++i) {
        if (l_col_ptr[i] < sym_c_ptr[i] || l_col_ptr[i] >= sym_c_ptr[i + 1] || sym_r_idx[l_col_ptr[i]] != i)
            return set_error(GLU_ERR_ARG, "invalid diagonal pointer of column %u", i);
        // rows strictly ascending in every column (the kernels search them)
        for (uint32_t p = sym_c_ptr[i] + 1; p < sym_c_ptr[i + 1]; ++p)
            if (sym_r_idx[p] <= sym_r_idx[p - 1])
                return set_error(GLU_ERR_ARG, "rows of column %u not strictly ascending", i);
    }
    for (uint32_t p = 0; p < nnz; ++p)
        if (sym_r_idx[p] >= n || csr_c_idx[p] >= n) return set_error(GLU_ERR_ARG, "row or column index out of range");
    // CSC positions of the CSR entries (rows ascending in every column)
    s.csr_pos.resize(nnz);
    {
        std::vector<uint32_t> fillp(s.csr_r_ptr.begin(), s.csr_r_ptr.end() - 1);
        for (uint32_t c = 0; c < n; ++c)
            for (uint32_t p = s.sym_c_ptr[c]; p < s.sym_c_ptr[c + 1]; ++p) {
                uint32_t r = s.sym_r_idx[p];
                uint32_t e = fillp[r]++;
                if (e >= s.csr_r_ptr[r + 1] || s.csr_c_idx[e] != c)
                    return set_error(GLU_ERR_ARG, "CSR arrays do not transpose the CSC pattern");
                s.csr_pos[e] = p;
            }
    }
    return create_handle(device, std::move(s), batch, out);
}

void glu_destroy(glu_handle_t h) {
    if (!h) return;
    DeviceGuard g(h->device);
    delete h;
}

glu_status glu_levels(glu_handle_t h, int32_t *num_lev, int32_t *level_ptr, int32_t *level_idx) {
    if (!h) return set_error(GLU_ERR_ARG, "null handle");
    if (num_lev) *num_lev = h->num_lev;
    if (level_ptr) memcpy(level_ptr, h->level_ptr.data(), sizeof(int32_t) * h->level_ptr.size());
    if (level_idx) memcpy(level_idx, h->level_idx.data(), sizeof(int32_t) * h->level_idx.size());
    return GLU_OK;
}

glu_status glu_set_transform(glu_handle_t h, const uint32_t *col_perm, const uint32_t *row_perm_inv,
                             const int32_t *pivot, const double *col_scale_perm, const double *row_scale,
                             int mc64_scale) {
    if (!h || !col_perm || !row_perm_inv || !pivot) return set_error(GLU_ERR_ARG, "null argument");
    if (mc64_scale && (!col_scale_perm || !row_scale)) return set_error(GLU_ERR_ARG, "null scale array");
    const uint32_t n = h->n;
    std::vector<uint32_t> in_idx(n), out_idx(n), tin_idx(n), tout_idx(n);
    std::vector<double> in_s(n), out_s(n), tin_s(n), tout_s(n);
    std::vector<uint32_t> cp_inv(n, UINT32_MAX), g(n, UINT32_MAX);
    for (uint32_t j = 0; j < n; ++j) {
        int32_t pj = pivot[j];
        if (pj < 0 || uint32_t(pj) >= n || col_perm[pj] >= n || row_perm_inv[j] >= n)
            return set_error(GLU_ERR_ARG, "permutation entry out of range");
        in_idx[j] = col_perm[pj];  // b[j] = rhs[rp[piv[j]]] * rows[piv[j]]
        in_s[j] = mc64_scale ? col_scale_perm[pj] : 1.0;
        out_idx[j] = row_perm_inv[j];  // x[j] = b[cp[j]] * cols[j]
        out_s[j] = mc64_scale ? row_scale[j] : 1.0;
        if (cp_inv[row_perm_inv[j]] != UINT32_MAX || g[in_idx[j]] != UINT32_MAX)
            return set_error(GLU_ERR_ARG, "permutation is not one-to-one");
        cp_inv[row_perm_inv[j]] = j;
        g[in_idx[j]] = j;
    }
    for (uint32_t i = 0; i < n; ++i) {
        tin_idx[i] = cp_inv[i];  // A^T: y[cp[j]] = b[j] * cols[j]
        tin_s[i] = out_s[cp_inv[i]];
        tout_idx[i] = g[i];  // x[rp[piv[j]]] = z[j] * rows[piv[j]]
        tout_s[i] = in_s[g[i]];
    }
    DeviceGuard gd(h->device);
    GLU_CUDA(upload(h->d_tr[0], in_idx), "upload transform");
    GLU_CUDA(upload(h->d_tr[2], out_idx), "upload transform");
    GLU_CUDA(upload(h->d_tr[4], tin_idx), "upload transform");
    GLU_CUDA(upload(h->d_tr[6], tout_idx), "upload transform");
    if (mc64_scale) {
        GLU_CUDA(upload(h->d_tr[1], in_s), "upload transform");
        GLU_CUDA(upload(h->d_tr[3], out_s), "upload transform");
        GLU_CUDA(upload(h->d_tr[5], tin_s), "upload transform");
        GLU_CUDA(upload(h->d_tr[7], tout_s), "upload transform");
    } else {
        for (int k = 1; k < 8; k += 2) h->d_tr[k].release();
    }
    h->T = TransformDev{h->d_tr[0].as<uint32_t>(), h->d_tr[1].as<double>(), h->d_tr[2].as<uint32_t>(),
                        h->d_tr[3].as<double>(),   h->d_tr[4].as<uint32_t>(), h->d_tr[5].as<double>(),
                        h->d_tr[6].as<uint32_t>(), h->d_tr[7].as<double>()};
    h->has_transform = true;
    return GLU_OK;
}

glu_status glu_set_source(glu_handle_t h, uint32_t nnz_src, const uint32_t *src_ap, const uint32_t *src_ai,
                          const uint32_t *src_slot, const double *src_scale) {
    if (!h || !src_ap || (nnz_src && (!src_ai || !src_slot))) return set_error(GLU_ERR_ARG, "null argument");
    const uint32_t n = h->n;
    if (src_ap[0] != 0 || src_ap[n] != nnz_src) return set_error(GLU_ERR_ARG, "inconsistent source pointers");
    std::vector<int64_t> lu_src(h->nnz, -1);
    std::vector<uint32_t> rcount(n + 1, 0);
    for (uint32_t c = 0; c < n; ++c) {
        if (src_ap[c] > src_ap[c + 1]) return set_error(GLU_ERR_ARG, "source pointers not monotone");
        for (uint32_t q = src_ap[c]; q < src_ap[c + 1]; ++q) {
            if (src_ai[q] >= n || src_slot[q] >= h->nnz) return set_error(GLU_ERR_ARG, "source entry out of range");
            if (lu_src[src_slot[q]] < 0) lu_src[src_slot[q]] = int64_t(q);
            rcount[src_ai[q] + 1]++;
        }
    }
    // CSR of A0 for the FP64 residual
    for (uint32_t r = 0; r < n; ++r) rcount[r + 1] += rcount[r];
    std::vector<uint32_t> rptr(rcount), cidx(nnz_src), vmap(nnz_src), ident(nnz_src);
    {
        std::vector<uint32_t> fillp(rcount.begin(), rcount.end() - 1);
        for (uint32_t c = 0; c < n; ++c)
            for (uint32_t q = src_ap[c]; q < src_ap[c + 1]; ++q) {
                uint32_t e = fillp[src_ai[q]]++;
                cidx[e] = c;
                vmap[e] = q;
            }
    }
    std::iota(ident.begin(), ident.end(), 0u);
    std::vector<double> scale(nnz_src, 1.0);
    if (src_scale) scale.assign(src_scale, src_scale + nnz_src);
    DeviceGuard g(h->device);
    GLU_CUDA(upload(h->d_src_lu, lu_src), "upload source");
    GLU_CUDA(upload(h->d_src_scale, scale), "upload source");
    GLU_CUDA(upload(h->d_a0_rptr, rptr), "upload source");
    GLU_CUDA(upload(h->d_a0_cidx, cidx), "upload source");
    GLU_CUDA(upload(h->d_a0_vmap, vmap), "upload source");
    GLU_CUDA(upload(h->d_a0_cptr, std::vector<uint32_t>(src_ap, src_ap + n + 1)), "upload source");
    GLU_CUDA(upload(h->d_a0_ridx, std::vector<uint32_t>(src_ai, src_ai + nnz_src)), "upload source");
    GLU_CUDA(upload(h->d_a0_ident, ident), "upload source");
    GLU_CUDA(h->d_ax0.alloc(sizeof(double) * std::max<size_t>(size_t(nnz_src) * h->batch, 1)), "allocate source values");
    h->nnz_src = nnz_src;
    h->has_source = true;
    h->ax0_loaded = false;
    return GLU_OK;
}

glu_status glu_load_lu_values(glu_handle_t h, uint32_t first, uint32_t count, const float *val,
                              glu_memory where, glu_stream stream) {
    if (!h || !val) return set_error(GLU_ERR_ARG, "null argument");
    Status s = check_range(h, first, count);
    if (s != GLU_OK) return s;
    DeviceGuard g(h->device);
    GLU_CUDA(cudaMemcpyAsync(h->d_val.as<float>() + size_t(first) * h->nnz, val,
                             sizeof(float) * size_t(h->nnz) * count,
                             where == GLU_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, S_(stream)),
             "copy values");
    if (where == GLU_HOST) GLU_CUDA(cudaStreamSynchronize(S_(stream)), "synchronize");
    h->factored = false;
    return GLU_OK;
}

glu_status glu_store_lu_values(glu_handle_t h, uint32_t first, uint32_t count, float *val,
                               glu_memory where, glu_stream stream) {
    if (!h || !val) return set_error(GLU_ERR_ARG, "null argument");
    Status s = check_range(h, first, count);
    if (s != GLU_OK) return s;
    DeviceGuard g(h->device);
    GLU_CUDA(cudaMemcpyAsync(val, h->d_val.as<float>() + size_t(first) * h->nnz,
                             sizeof(float) * size_t(h->nnz) * count,
                             where == GLU_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, S_(stream)),
             "copy values");
    if (where == GLU_HOST) GLU_CUDA(cudaStreamSynchronize(S_(stream)), "synchronize");
    return GLU_OK;
}

glu_status glu_load_source_values(glu_handle_t h, uint32_t first, uint32_t count, const double *ax0,
                                  glu_memory where, glu_stream stream) {
    if (!h || !ax0) return set_error(GLU_ERR_ARG, "null argument");
    if (!h->has_source) return set_error(GLU_ERR_STATE, "no source matrix set (glu_set_source)");
    Status s = check_range(h, first, count);
    if (s != GLU_OK) return s;
    DeviceGuard g(h->device);
    cudaStream_t st = S_(stream);
    double *dst = h->d_ax0.as<double>() + size_t(first) * h->nnz_src;
    GLU_CUDA(cudaMemcpyAsync(dst, ax0, sizeof(double) * size_t(h->nnz_src) * count,
                             where == GLU_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, st),
             "copy source values");
    GLU_CUDA(launch_gather_values(h->d_src_lu.as<int64_t>(), dst, h->nnz_src, h->d_src_scale.as<double>(),
                                  h->nnz, h->d_val.as<float>() + size_t(first) * h->nnz, h->nnz, count, st),
             "place values");
    if (where == GLU_HOST) GLU_CUDA(cudaStreamSynchronize(st), "synchronize");
    h->ax0_loaded = true;
    h->factored = false;
    return GLU_OK;
}

}  // extern "C"

namespace {

// Everything of a factorization up to its last launch, on st; the status word
// (and the perturbation of value set `first`) are copied to pinned memory
// asynchronously.  factor_finish reads them once st has completed.
Status factor_enqueue(glu_handle_s *h, uint32_t first, uint32_t count, int perturb, cudaStream_t st) {
    Status s = GLU_OK;
    float *val = h->d_val.as<float>() + size_t(first) * h->nnz;
    const uint64_t stride = h->nnz;
    const float *pert = nullptr;
    GLU_CUDA(cudaMemsetAsync(h->d_status.p, 0, sizeof(uint32_t), st), "reset status");
    GLU_CUDA(cudaEventRecord(h->ev0, st), "event");
    KernelProfiler &pf = h->prof;
    pf.used = 0;
    uint64_t nlaunch = 0;  // kernel launches of this call
#define GLU_LAUNCH(kind, call, what)                    \
    do {                                                \
        GLU_CUDA(pf.begin(st), "profile event");        \
        GLU_CUDA((call), (what));                       \
        ++nlaunch;                                      \
        GLU_CUDA(pf.end((kind), st), "profile event");  \
    } while (0)
    if (perturb) {
        GLU_LAUNCH(KK_PERT, launch_pert(h->P, val, stride, count, h->d_colmax.as<float>(), h->d_pert.as<float>() + first, st),
                   "perturbation");
        pert = h->d_pert.as<float>() + first;
    }
    const uint32_t NL = h->use_sn ? 0u : uint32_t(h->levels_h.size());
    if (h->use_sn) {
        for (const SnLevel &lv : h->sn_levels) {
            if (lv.dblocks)
                GLU_LAUNCH(KK_SN_DIAG, launch_sn_diag(h->P, h->SN, val, stride, count, pert, lv.db0, lv.dblocks, st),
                           "factor (supernode diagonal blocks)");
            if (lv.pblocks)
                GLU_LAUNCH(KK_SN_PANEL,
                           launch_sn_panel(h->P, h->SN, val, stride, count, pert, lv.pb0, lv.pblocks, lv.panel_w, st),
                           "factor (supernode panels)");
            if (lv.ublocks)
                GLU_LAUNCH(KK_SN_UPDATE,
                           launch_sn_update(h->P, h->SN, val, stride, count, lv.ub0, lv.ublocks, lv.atomic,
                                            h->tune.batch_tile, st),
                           "factor (supernode updates)");
        }
    }
    for (const Step &stp : (h->use_sn ? std::vector<Step>() : h->steps)) {
        if (stp.kind == STEP_CHAIN) {
            GLU_LAUNCH(KK_CHAIN,
                       launch_factor_chain(h->P, h->F, val, stride, count, pert, stp.l0, stp.l1, h->chain_cluster, st),
                       "factor (narrow levels)");
        } else {
            const LevelInfo &cur = h->levels_h[stp.l0];
            const LevelInfo *prev = stp.l0 > 0 ? &h->levels_h[stp.l0 - 1] : nullptr;
            GLU_LAUNCH(KK_LEVEL,
                       launch_factor_level(h->P, h->F, val, stride, count, pert, cur, prev, h->items_h[stp.l0], st),
                       "factor (level)");
        }
    }
    if (NL)
        GLU_LAUNCH(KK_SCALE, launch_scale_level(h->P, h->F, val, stride, count, pert, h->levels_h[NL - 1], st),
                   "factor (scale)");
    // dense trailing block: in place, or through the dense buffer
    float *dbase = h->dense_buffer ? h->d_dense.as<float>() + size_t(first) * h->m * h->m : val;
    const uint64_t dstride = h->dense_buffer ? uint64_t(h->m) * h->m : stride;
    if (h->m && h->dense_buffer)
        GLU_LAUNCH(KK_DGATHER,
                   launch_dense_gather(h->P, val, stride, count, h->t, h->m, h->d_tail_start.as<uint32_t>(), dbase, st),
                   "factor (dense gather)");
    // Small trailing blocks: panel, update, one panel at a time.  Large ones
    // (tune.dense_lookahead columns or more) take the panels in groups of
    // tune.dense_group: panel k0, then for each further panel j of the group
    // its row and column strips updated by panels 0 .. j - 1 (K = 64 j) and
    // panel j itself, then one update of the rest with the whole group (K =
    // 64 x group: every entry still receives its products in column order,
    // C read and written once per group).  The panels and the strips run on a
    // high-priority internal stream, the rest of the group's update on st,
    // concurrently with the next group's first panel, which it does not touch;
    // the next strips wait for it (the same entries, updated in column order).
    const bool lookahead = h->aux && h->tune.dense_lookahead && h->m >= h->tune.dense_lookahead && h->m > kDenseNB;
    const uint32_t *doff = h->d_doff.as<uint32_t>();
    float *dscr = h->d_diag_scratch.as<float>();
    cudaStream_t ps = lookahead ? h->aux : st;  // panels and strips
    bool rest_pending = false;
    const uint32_t nb = kDenseNB;
    // tensor-core updates for wide trailing blocks; their operand packs are
    // allocated once per handle
    const bool tc = h->m && h->tune.dense_tc_min && h->m >= h->tune.dense_tc_min;
    if (tc && h->pack_m != h->m) {
        const size_t pack_bytes = sizeof(uint16_t) * kDensePackRow * size_t(h->m) * h->batch;
        GLU_CUDA(h->d_packA.alloc(pack_bytes), "allocate tensor-core operand packs");
        GLU_CUDA(h->d_packB.alloc(pack_bytes), "allocate tensor-core operand packs");
        GLU_CUDA(dense_tc_tensor_map(h->d_packA.as<uint16_t>(), h->m, h->batch, &h->map_packA), "tensor map");
        GLU_CUDA(dense_tc_tensor_map(h->d_packB.as<uint16_t>(), h->m, h->batch, &h->map_packB), "tensor map");
        GLU_CUDA(h->d_tc_counter.alloc(sizeof(uint32_t) * 2), "allocate tile counters");
        h->pack_m = h->m;
    }
    uint32_t *dstatus = h->d_status.as<uint32_t>();
    double upd_bytes = 0, upd_flops = 0;
    // The sparse columns' deferred updates of the block (the plan has them
    // only when the block updates on the tensor cores): per group of up to 128
    // columns, their tail rows of L and tail columns of U into the packs, then
    // A22 -= L U over the whole block.
    if (tc && !h->couple_groups.empty()) {
        const double mm = h->m;
        for (const CoupleGroup &gr : h->couple_groups) {
            const uint32_t nc = gr.c1 - gr.c0;
            GLU_LAUNCH(KK_COUPLE_PACK,
                       launch_couple_pack(h->P, val, stride, count, h->t, h->m, nc, gr.c0,
                                          h->d_couple_lstart.as<uint32_t>(), h->d_couple_ustart.as<uint32_t>(),
                                          h->d_packA.as<uint16_t>(), h->d_packB.as<uint16_t>(), st),
                       "factor (coupling pack)");
            GLU_LAUNCH(KK_UPDATE_TC,
                       launch_couple_update_tc(h->map_packA, h->map_packB, dbase, dstride, count, doff, h->m, nc,
                                               dstatus, h->spin_limit, h->num_sms, h->d_tc_counter.as<uint32_t>(), st),
                       "factor (coupling update)");
            upd_bytes += double(count) * (8.0 * mm * mm + 8.0 * nc * mm);
            upd_flops += double(count) * 2.0 * nc * mm * mm;
        }
    }
    if (lookahead) {
        GLU_CUDA(cudaEventRecord(h->ev_fork, st), "event");
        GLU_CUDA(cudaStreamWaitEvent(ps, h->ev_fork, 0), "stream wait");
    }
    // A region goes to the tensor cores when its area over all value sets
    // reaches two 128 x 128 tiles per SM, or dense_tc_min^2 entries if less;
    // thinner ones (the look-ahead strips, the last small updates) stay on the
    // FP32 FMA kernel, whose launch costs less than the tensor-core kernel's
    // set-up.
    const uint64_t tc_area = std::min<uint64_t>(uint64_t(2) * h->num_sms * kTcTile * kTcTile,
                                                uint64_t(h->tune.dense_tc_min) * h->tune.dense_tc_min);
    auto tc_region = [&](uint32_t rows, uint32_t cols) { return tc && uint64_t(rows) * cols * count >= tc_area; };
    auto update = [&](uint32_t k0, uint32_t kb, DenseRegion reg, cudaStream_t s) -> cudaError_t {
        const uint32_t nr = reg.r_hi > reg.r_lo ? reg.r_hi - reg.r_lo : 0;
        const uint32_t nc = reg.c_hi > reg.c_lo ? reg.c_hi - reg.c_lo : 0;
        const double rows = nr, cols = nc;
        upd_bytes += double(count) * (8.0 * rows * cols + 4.0 * kb * (rows + cols));
        upd_flops += double(count) * 2.0 * kb * rows * cols;
        cudaError_t e = pf.begin(s);
        if (e != cudaSuccess) return e;
        if (tc_region(nr, nc)) {
            // a tile counter per stream (launches on one stream run in order)
            uint32_t *ctr = h->d_tc_counter.as<uint32_t>() + (s == st ? 0 : 1);
            e = launch_dense_update_tc(h->map_packA, h->map_packB, dbase, dstride, count, doff, h->m, k0, kb, dscr,
                                       reg, dstatus, h->spin_limit, h->num_sms, ctr, s);
            if (e == cudaSuccess) e = pf.end(KK_UPDATE_TC, s);
        } else {
            e = launch_dense_update(dbase, dstride, count, doff, h->m, k0, kb, dscr, reg, s);
            if (e == cudaSuccess) e = pf.end(KK_UPDATE, s);
        }
        ++nlaunch;
        return e;
    };
    // BF16 three-part operands of panel k0 (slot0 = 64 j for panel j of a
    // look-ahead group), on the panel stream
    auto pack = [&](uint32_t k0, uint32_t kb, uint32_t slot0, bool needed) -> cudaError_t {
        if (!needed) return cudaSuccess;
        cudaError_t e = pf.begin(ps);
        if (e == cudaSuccess)
            e = launch_dense_pack(dbase, dstride, count, doff, h->m, k0, kb, slot0, h->d_packA.as<uint16_t>(),
                                  h->d_packB.as<uint16_t>(), ps);
        if (e == cudaSuccess) e = pf.end(KK_PACK, ps);
        ++nlaunch;
        return e;
    };
    auto panel = [&](uint32_t k0, uint32_t kb) -> cudaError_t {
        cudaError_t e = pf.begin(ps);
        if (e == cudaSuccess)
            e = launch_dense_panel(dbase, dstride, count, doff, h->m, k0, kb, pert, dscr, 0, h->num_sms, ps);
        if (e == cudaSuccess) e = pf.end(KK_PANEL, ps);
        nlaunch += dense_panel_launches(count, h->m, k0, kb, h->num_sms);
        return e;
    };
    // panels per look-ahead group: the group's rest takes K = 64 x group
    const uint32_t group = lookahead ? std::min<uint32_t>(std::max<uint32_t>(h->tune.dense_group, 2u),
                                                          kDenseGroupMax)
                                     : 1u;
    for (uint32_t k0 = 0; k0 < h->m;) {
        const uint32_t kb0 = std::min<uint32_t>(nb, h->m - k0);
        const uint32_t rest0 = h->m - (k0 + kb0);
        GLU_CUDA(panel(k0, kb0), "factor (dense panel)");
        if (rest_pending) {
            GLU_CUDA(cudaStreamWaitEvent(ps, h->ev_rest, 0), "stream wait");
            rest_pending = false;
        }
        // panels of this group: all but the last are full width
        const uint32_t g = std::min<uint32_t>(group, (h->m - k0 + nb - 1) / nb);
        // packs are written when any update of this group may read them: every
        // region of the group lies in the trailing block from k0 on
        const bool packed = tc_region(h->m - k0, h->m - k0);
        // after the previous group's update, which reads the packs
        GLU_CUDA(pack(k0, kb0, 0, packed), "factor (dense pack)");
        if (g == 1) {  // small trailing blocks, last panels: plain steps
            GLU_CUDA(update(k0, kb0, DenseRegion{0, rest0, 0, rest0, 1, k0}, ps), "factor (dense update)");
            k0 += kb0;
            continue;
        }
        // panel j of the group: its row and column strips take the updates of
        // panels 0 .. j - 1 (K = 64 j; the first launch after panel j - 1
        // writes its diagonal block back), then the panel itself
        uint32_t kk = kb0;  // K of the group so far
        for (uint32_t j = 1; j < g; ++j) {
            const uint32_t kj = k0 + kk, kbj = std::min<uint32_t>(nb, h->m - kj), tj = h->m - kj;
            const uint32_t hj = std::min<uint32_t>(nb, tj);
            GLU_CUDA(update(k0, kk, DenseRegion{0, hj, 0, tj, 1, kj - nb}, ps), "factor (dense update)");
            if (tj > hj) GLU_CUDA(update(k0, kk, DenseRegion{hj, tj, 0, hj, 0, kj - nb}, ps), "factor (dense update)");
            GLU_CUDA(panel(kj, kbj), "factor (dense panel)");
            GLU_CUDA(pack(kj, kbj, kDenseNB * j, packed), "factor (dense pack)");
            kk += kbj;
        }
        // the rest with the whole group (K = kk): the next group's first panel
        // strips on the panel stream, the remainder on st concurrently with
        // that panel
        const uint32_t kl = k0 + kk - std::min<uint32_t>(nb, kk - (g - 1) * nb);  // last panel of the group
        const uint32_t rest1 = h->m - (k0 + kk);
        if (rest1 <= nb) {
            GLU_CUDA(update(k0, kk, DenseRegion{0, rest1, 0, rest1, 1, kl}, ps), "factor (dense update)");
        } else {
            GLU_CUDA(cudaEventRecord(h->ev_panel, ps), "event");
            GLU_CUDA(update(k0, kk, DenseRegion{0, nb, 0, rest1, 1, kl}, ps), "factor (dense update)");
            GLU_CUDA(update(k0, kk, DenseRegion{nb, rest1, 0, nb, 0, kl}, ps), "factor (dense update)");
            GLU_CUDA(cudaStreamWaitEvent(st, h->ev_panel, 0), "stream wait");
            GLU_CUDA(update(k0, kk, DenseRegion{nb, rest1, nb, rest1, 0, kl}, st), "factor (dense update)");
            GLU_CUDA(cudaEventRecord(h->ev_rest, st), "event");
            rest_pending = true;
        }
        k0 += kk;
    }
    if (lookahead) {
        if (rest_pending) GLU_CUDA(cudaStreamWaitEvent(ps, h->ev_rest, 0), "stream wait");
        GLU_CUDA(cudaEventRecord(h->ev_fork, ps), "event");
        GLU_CUDA(cudaStreamWaitEvent(st, h->ev_fork, 0), "stream wait");
    }
    if (h->m && h->dense_buffer)
        GLU_LAUNCH(KK_DSCATTER,
                   launch_dense_scatter(h->P, val, stride, count, h->t, h->m, h->d_tail_start.as<uint32_t>(), dbase, st),
                   "factor (dense scatter)");
    if (h->m) {
        GLU_CUDA(h->d_dinv.ensure(sizeof(float) * dinv_per_set(h) * h->batch), "allocate diagonal-block inverses");
        GLU_LAUNCH(KK_DIAG_INV,
                   launch_dense_diag_inv(dbase, dstride, count, doff, h->m,
                                         h->d_dinv.as<float>() + size_t(first) * dinv_per_set(h), st),
                   "factor (diagonal-block inverses)");
    }
    GLU_LAUNCH(KK_CHECK, launch_check_pivots(h->P, val, stride, count, h->d_status.as<uint32_t>(), st), "pivot check");
#undef GLU_LAUNCH
    GLU_CUDA(cudaEventRecord(h->ev1, st), "event");
    GLU_CUDA(cudaMemcpyAsync(h->h_status, h->d_status.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, st),
             "read status");
    if (perturb)
        GLU_CUDA(cudaMemcpyAsync(h->h_status + 1, h->d_pert.as<float>() + first, sizeof(float),
                                 cudaMemcpyDeviceToHost, st),
                 "read perturbation");
    h->pending_launches = nlaunch;
    h->pending_upd_bytes = upd_bytes;
    h->pending_upd_flops = upd_flops;
    return s;
}

// The host half of a factorization whose stream has completed: status,
// statistics, per-kernel times.
Status factor_finish(glu_handle_s *h, int perturb) {
    const uint32_t flags = h->h_status[0];
    h->prof.collect();
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->stats.last_factor_ms = ms;
    h->stats.factor_launches = h->pending_launches;
    h->stats.dense_update_bytes = h->pending_upd_bytes;
    h->stats.dense_update_flops = h->pending_upd_flops;
    if (perturb) std::memcpy(&h->stats.pert, h->h_status + 1, sizeof(float));
    h->factored = true;
    if (flags & DEV_TIMEOUT) return set_error(GLU_ERR_TIMEOUT, "factorization wait timed out");
    if (flags & (DEV_ZERO_PIVOT | DEV_NONFINITE_PIVOT))
        return set_error(GLU_ERR_SINGULAR, "%s pivot encountered", (flags & DEV_ZERO_PIVOT) ? "zero" : "non-finite");
    return GLU_OK;
}

}  // namespace

extern "C" {

glu_status glu_factor(glu_handle_t h, uint32_t first, uint32_t count, int perturb, glu_stream stream) {
    TraceRange trace_("glu_factor");
    if (!h) return set_error(GLU_ERR_ARG, "null handle");
    Status s = check_range(h, first, count);
    if (s != GLU_OK) return s;
    DeviceGuard g(h->device);
    cudaStream_t st = S_(stream);
    s = factor_enqueue(h, first, count, perturb, st);
    if (s != GLU_OK) return s;
    GLU_CUDA(cudaStreamSynchronize(st), "synchronize");
    return factor_finish(h, perturb);
}

glu_status glu_factor_many(uint32_t count, const glu_handle_t *handles, int perturb, const glu_stream *streams,
                           uint32_t nstreams) {
    TraceRange trace_("glu_factor_many");
    if (count == 0) return GLU_OK;
    if (!handles || (nstreams && !streams)) return set_error(GLU_ERR_ARG, "null argument");
    for (uint32_t i = 0; i < count; ++i)
        if (!handles[i]) return set_error(GLU_ERR_ARG, "null handle %u", i);
    auto stream_of = [&](uint32_t i) { return nstreams ? S_(streams[i % nstreams]) : cudaStream_t(nullptr); };
    // every system's launches first, each on its stream ...
    for (uint32_t i = 0; i < count; ++i) {
        glu_handle_s *h = handles[i];
        DeviceGuard g(h->device);
        Status s = factor_enqueue(h, 0, h->batch, perturb, stream_of(i));
        if (s != GLU_OK) return set_error(s, "system %u: %s", i, glu_last_error());
    }
    // ... then one wait per stream, then every system's status
    for (uint32_t i = 0; i < std::max<uint32_t>(nstreams, 1) && i < count; ++i) {
        DeviceGuard g(handles[i]->device);
        GLU_CUDA(cudaStreamSynchronize(stream_of(i)), "synchronize");
    }
    Status first_err = GLU_OK;
    std::string msg;
    for (uint32_t i = 0; i < count; ++i) {
        Status s = factor_finish(handles[i], perturb);
        if (s != GLU_OK && first_err == GLU_OK) {
            first_err = s;
            msg = "system " + std::to_string(i) + ": " + glu_last_error();
        }
    }
    if (first_err != GLU_OK) return set_error(first_err, "%s", msg.c_str());
    return GLU_OK;
}

glu_status glu_solve(glu_handle_t h, uint32_t inst, uint32_t nrhs, const float *b, float *x,
                     glu_memory where, glu_stream stream) {
    TraceRange trace_("glu_solve");
    if (!h) return set_error(GLU_ERR_ARG, "null handle");
    return solve_f32(h, inst, nrhs, b, x, where, false, S_(stream));
}

glu_status glu_solve_transposed(glu_handle_t h, uint32_t inst, uint32_t nrhs, const float *b, float *x,
                                glu_memory where, glu_stream stream) {
    if (!h) return set_error(GLU_ERR_ARG, "null handle");
    return solve_f32(h, inst, nrhs, b, x, where, true, S_(stream));
}

}  // extern "C"

namespace {

// A refined solve of value sets [first, first + count) of one handle, run as
// a sequence of enqueued steps so that many of them (glu_solve_refined_many)
// can advance together with one host synchronisation per step.
struct RefineJob {
    glu_handle_s *h = nullptr;
    uint32_t first = 0, count = 0, nrhs = 0;
    const double *b = nullptr;
    double *x = nullptr;
    double tol = 0;
    uint32_t maxit = 0;
    bool tr = false, host = false;
    cudaStream_t st = nullptr;
    // state
    uint32_t nvec = 0, it = 0;
    size_t len = 0;
    const double *bz = nullptr;
    double *xz = nullptr;
    double worst2 = 0, worstinf = 0;
    bool done = false;
};

Status refine_prepare(RefineJob &j) {
    glu_handle_s *h = j.h;
    if (!h->factored) return set_error(GLU_ERR_STATE, "solve before factorization");
    if (!h->has_source || !h->ax0_loaded)
        return set_error(GLU_ERR_STATE, "refinement needs the source matrix values (glu_load_source_values)");
    if (uint64_t(j.nrhs) * j.count > 65535)
        return set_error(GLU_ERR_UNSUPPORTED, "count * nrhs = %llu right-hand sides exceed 65,535 per call",
                         (unsigned long long)j.nrhs * j.count);
    j.nvec = j.nrhs * j.count;
    j.len = size_t(h->n) * j.nvec;
    GLU_CUDA(h->d_y.ensure(sizeof(float) * j.len), "allocate");
    GLU_CUDA(h->d_b64.ensure(sizeof(double) * j.len * (j.host ? 1 : 0) + 8), "allocate");
    GLU_CUDA(h->d_x64.ensure(sizeof(double) * j.len * (j.host ? 1 : 0) + 8), "allocate");
    GLU_CUDA(h->d_r64.ensure(sizeof(double) * j.len), "allocate");
    GLU_CUDA(h->d_norms.ensure(sizeof(double) * 4 * j.nvec), "allocate");
    if (h->h_norms_cap < 4 * size_t(j.nvec)) {
        if (h->h_norms) cudaFreeHost(h->h_norms);
        h->h_norms = nullptr;
        h->h_norms_cap = 0;
        GLU_CUDA(cudaMallocHost(reinterpret_cast<void **>(&h->h_norms), sizeof(double) * 4 * j.nvec),
                 "allocate pinned");
        h->h_norms_cap = 4 * size_t(j.nvec);
    }
    return GLU_OK;
}

// r = b - A0 x for every vector, norms to the host (asynchronously).
Status refine_residual(RefineJob &j) {
    glu_handle_s *h = j.h;
    const uint32_t *rptr = j.tr ? h->d_a0_cptr.as<uint32_t>() : h->d_a0_rptr.as<uint32_t>();
    const uint32_t *cidx = j.tr ? h->d_a0_ridx.as<uint32_t>() : h->d_a0_cidx.as<uint32_t>();
    const uint32_t *vmap = j.tr ? h->d_a0_ident.as<uint32_t>() : h->d_a0_vmap.as<uint32_t>();
    const double *ax0 = h->d_ax0.as<double>() + size_t(j.first) * h->nnz_src;
    double *norms = h->d_norms.as<double>();
    h->stats.solve_launches += 1;
    GLU_CUDA(launch_residual(rptr, cidx, vmap, ax0, h->n, j.bz, j.xz, h->d_r64.as<double>(), j.nvec, j.nrhs,
                             h->nnz_src, norms, j.st),
             "residual");
    GLU_CUDA(cudaMemcpyAsync(h->h_norms, norms, sizeof(double) * 4 * j.nvec, cudaMemcpyDeviceToHost, j.st),
             "read norms");
    return GLU_OK;
}

// x = solve(v) (accumulate: x += solve(v)) for every vector v of src.
Status refine_solve(RefineJob &j, const double *src, int accumulate) {
    glu_handle_s *h = j.h;
    const TransformDev &T = h->T;
    float *y = h->d_y.as<float>();
    h->stats.solve_launches += 2;  // the two transforms
    GLU_CUDA(launch_transform_f64_to_f32(j.tr ? T.tin_idx : T.in_idx, j.tr ? T.tin_scale : T.in_scale, src, y, h->n,
                                         j.nvec, j.st),
             "transform");
    Status s = solve_inplace(h, j.first, j.count, y, j.nrhs, j.tr, j.st);
    if (s != GLU_OK) return s;
    GLU_CUDA(launch_transform_f32_to_f64_add(j.tr ? T.tout_idx : T.out_idx, j.tr ? T.tout_scale : T.out_scale, y,
                                             j.xz, h->n, j.nvec, accumulate, j.st),
             "transform");
    return GLU_OK;
}

// Enqueues x0 = solve(b) and the first residual.
Status refine_start(RefineJob &j) {
    glu_handle_s *h = j.h;
    if (j.host) {
        GLU_CUDA(cudaMemcpyAsync(h->d_b64.p, j.b, sizeof(double) * j.len, cudaMemcpyHostToDevice, j.st), "copy b");
        j.bz = h->d_b64.as<double>();
        j.xz = h->d_x64.as<double>();
    } else {
        j.bz = j.b;
        j.xz = j.x;
    }
    double *norms = h->d_norms.as<double>();
    GLU_CUDA(cudaMemsetAsync(h->d_status.p, 0, sizeof(uint32_t), j.st), "reset status");
    h->stats.solve_launches = 1;  // the norms of b; every solve and residual adds its own
    GLU_CUDA(launch_norms(j.bz, h->n, j.nvec, norms + 2 * j.nvec, j.st), "norms");
    Status s = refine_solve(j, j.bz, 0);
    if (s != GLU_OK) return s;
    return refine_residual(j);
}

// After the stream has completed the last residual: stop, or enqueue
// x += solve(r) and the next residual.
Status refine_step(RefineJob &j) {
    glu_handle_s *h = j.h;
    const double *hn = h->h_norms;
    j.worst2 = 0;
    j.worstinf = 0;
    for (uint32_t v = 0; v < j.nvec; ++v) {
        double bn2 = std::sqrt(hn[2 * j.nvec + 2 * v]), bninf = hn[2 * j.nvec + 2 * v + 1];
        double rn2 = std::sqrt(hn[2 * v]), rninf = hn[2 * v + 1];
        double rel2 = bn2 > 0 ? rn2 / bn2 : rn2, relinf = bninf > 0 ? rninf / bninf : rninf;
        if (!(rel2 == rel2)) rel2 = INFINITY;
        j.worst2 = std::max(j.worst2, rel2);
        j.worstinf = std::max(j.worstinf, relinf);
    }
    if (j.worst2 <= j.tol || j.it >= j.maxit) {
        j.done = true;
        if (j.host)
            GLU_CUDA(cudaMemcpyAsync(j.x, j.xz, sizeof(double) * j.len, cudaMemcpyDeviceToHost, j.st), "copy x");
        GLU_CUDA(cudaMemcpyAsync(h->h_status, h->d_status.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, j.st),
                 "read status");
        return GLU_OK;
    }
    ++j.it;
    Status s = refine_solve(j, h->d_r64.as<double>(), 1);
    if (s != GLU_OK) return s;
    return refine_residual(j);
}

// After the stream has completed the job's last step.
Status refine_finish(RefineJob &j, glu_refine_stats *stats) {
    if (j.h->h_status[0] & DEV_TIMEOUT) return set_error(GLU_ERR_TIMEOUT, "solve dependency wait timed out");
    if (stats) *stats = glu_refine_stats{j.it, j.worst2, j.worstinf};
    if (!(j.worst2 <= j.tol))
        return set_error(GLU_ERR_NOT_CONVERGED, "refinement stopped at relative residual %.3e > %.3e", j.worst2,
                         j.tol);
    return GLU_OK;
}

}  // namespace

extern "C" {

glu_status glu_solve_refined(glu_handle_t h, uint32_t first, uint32_t count, uint32_t nrhs,
                             const double *b, double *x, double tol, uint32_t maxit, int transposed,
                             glu_memory where, glu_refine_stats *stats, glu_stream stream) {
    TraceRange trace_("glu_solve_refined");
    if (!h || !b || !x) return set_error(GLU_ERR_ARG, "null argument");
    Status s = check_range(h, first, count);
    if (s != GLU_OK) return s;
    if (nrhs == 0) return GLU_OK;
    DeviceGuard g(h->device);
    RefineJob j;
    j.h = h;
    j.first = first;
    j.count = count;
    j.nrhs = nrhs;
    j.b = b;
    j.x = x;
    j.tol = tol;
    j.maxit = maxit;
    j.tr = transposed != 0;
    j.host = where == GLU_HOST;
    j.st = S_(stream);
    if ((s = refine_prepare(j)) != GLU_OK || (s = refine_start(j)) != GLU_OK) return s;
    // every value set in each step, until the worst relative residual of all
    // right-hand sides meets tol (one synchronisation per step)
    while (!j.done) {
        GLU_CUDA(cudaStreamSynchronize(j.st), "synchronize");
        if ((s = refine_step(j)) != GLU_OK) return s;
    }
    GLU_CUDA(cudaStreamSynchronize(j.st), "synchronize");
    return refine_finish(j, stats);
}

glu_status glu_solve_refined_many(uint32_t count, const glu_handle_t *handles, const uint32_t *nrhs,
                                  const double *const *b, double *const *x, double tol, uint32_t maxit,
                                  glu_memory where, glu_refine_stats *stats, const glu_stream *streams,
                                  uint32_t nstreams) {
    TraceRange trace_("glu_solve_refined_many");
    if (count == 0) return GLU_OK;
    if (!handles || !nrhs || !b || !x || (nstreams && !streams)) return set_error(GLU_ERR_ARG, "null argument");
    std::vector<RefineJob> jobs(count);
    for (uint32_t i = 0; i < count; ++i) {
        if (!handles[i] || !b[i] || !x[i]) return set_error(GLU_ERR_ARG, "null argument of system %u", i);
        RefineJob &j = jobs[i];
        j.h = handles[i];
        j.first = 0;
        j.count = j.h->batch;
        j.nrhs = nrhs[i];
        j.b = b[i];
        j.x = x[i];
        j.tol = tol;
        j.maxit = maxit;
        j.host = where == GLU_HOST;
        j.st = nstreams ? S_(streams[i % nstreams]) : nullptr;
        j.done = j.nrhs == 0;
    }
    auto fail = [&](uint32_t i, Status s) { return set_error(s, "system %u: %s", i, glu_last_error()); };
    for (uint32_t i = 0; i < count; ++i) {
        if (jobs[i].done) continue;
        DeviceGuard g(jobs[i].h->device);
        Status s = refine_prepare(jobs[i]);
        if (s == GLU_OK) s = refine_start(jobs[i]);
        if (s != GLU_OK) return fail(i, s);
    }
    const uint32_t nsync = std::max<uint32_t>(std::min(nstreams, count), 1);
    for (;;) {
        bool pending = false;
        for (uint32_t i = 0; i < count; ++i) pending |= !jobs[i].done;
        for (uint32_t k = 0; k < nsync; ++k) {
            DeviceGuard g(jobs[k].h->device);
            GLU_CUDA(cudaStreamSynchronize(jobs[k].st), "synchronize");
        }
        if (!pending) break;
        for (uint32_t i = 0; i < count; ++i) {
            if (jobs[i].done) continue;
            DeviceGuard g(jobs[i].h->device);
            Status s = refine_step(jobs[i]);
            if (s != GLU_OK) return fail(i, s);
        }
    }
    Status first_err = GLU_OK;
    std::string msg;
    for (uint32_t i = 0; i < count; ++i) {
        if (jobs[i].nrhs == 0) continue;
        Status s = refine_finish(jobs[i], stats ? stats + i : nullptr);
        if (s != GLU_OK && first_err == GLU_OK) {
            first_err = s;
            msg = "system " + std::to_string(i) + ": " + glu_last_error();
        }
    }
    if (first_err != GLU_OK) return set_error(first_err, "%s", msg.c_str());
    return GLU_OK;
}

glu_status glu_get_stats(glu_handle_t h, glu_stats *stats) {
    if (!h || !stats) return set_error(GLU_ERR_ARG, "null argument");
    *stats = h->stats;
    return GLU_OK;
}

glu_status glu_profile_enable(glu_handle_t h, int on) {
    if (!h) return set_error(GLU_ERR_ARG, "null handle");
    h->prof.on = on != 0;
    h->prof.used = 0;
    return GLU_OK;
}

glu_status glu_kernel_times(glu_handle_t h, float *ms, uint32_t *launches) {
    if (!h) return set_error(GLU_ERR_ARG, "null handle");
    for (int k = 0; k < GLU_KERNEL_KINDS; ++k) {
        if (ms) ms[k] = h->prof.ms[k];
        if (launches) launches[k] = h->prof.n[k];
    }
    return GLU_OK;
}

const char *glu_kernel_kind_name(int kind) {
    return (kind >= 0 && kind < GLU_KERNEL_KINDS) ? kKindNames[kind] : "";
}

glu_status glu_set_wait_limit(glu_handle_t h, uint32_t polls) {
    if (!h) return set_error(GLU_ERR_ARG, "null handle");
    h->spin_limit = polls ? polls : kSpinLimit;
    h->S.spin_limit = h->spin_limit;
    return GLU_OK;
}

glu_status glu_debug_inject(glu_handle_t h, int what, uint32_t value) {
    switch (what) {
        case GLU_INJECT_ALLOC_FAILURES:
            g_fail_allocs.store(int(std::min<uint32_t>(value, 1u << 30)), std::memory_order_relaxed);
            return GLU_OK;
        case GLU_INJECT_UNSET_SOLVE_FLAG:
            if (!h) return set_error(GLU_ERR_ARG, "null handle");
            if (h->m == 0) return set_error(GLU_ERR_UNSUPPORTED, "the factorization has no dense trailing block");
            h->inject_unset_flag = true;
            return GLU_OK;
        default:
            return set_error(GLU_ERR_ARG, "unknown injection %d", what);
    }
}

glu_status glu_get_tuning(glu_handle_t h, glu_tuning *t) {
    if (!h || !t) return set_error(GLU_ERR_ARG, "null argument");
    *t = h->tune;
    return GLU_OK;
}

glu_status glu_set_tuning(glu_handle_t h, const glu_tuning *t) {
    if (!h || !t) return set_error(GLU_ERR_ARG, "null argument");
    if (t->group_lanes && (t->group_lanes < 4 || t->group_lanes > 32 || (t->group_lanes & (t->group_lanes - 1))))
        return set_error(GLU_ERR_ARG, "group_lanes must be 0 or a power of two in [4, 32]");
    if (t->chain_cluster > 16) return set_error(GLU_ERR_ARG, "chain_cluster must be <= 16");
    if (t->solve_cluster > 16) return set_error(GLU_ERR_ARG, "solve_cluster must be <= 16");
    if (t->dense_group < 2 || t->dense_group > kDenseGroupMax)
        return set_error(GLU_ERR_ARG, "dense_group must be in [2, %u]", kDenseGroupMax);
    DeviceGuard g(h->device);
    h->tune = *t;
    if (h->tune.chain_cluster) h->chain_cluster = h->tune.chain_cluster;
    Status s = build_plan(h);
    h->factored = false;
    return s;
}

}  // extern "C"
