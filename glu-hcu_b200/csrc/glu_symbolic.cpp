// Host symbolic phase: the L+U fill pattern, its CSR transpose and the
// placement of A's values into the pattern.
//
// Output layout and contents are those of the reference's Symbolic_Matrix
// (include/symbolic.h:9-51): CSC sym_c_ptr / sym_r_idx with rows ascending in
// every column and l_col_ptr the position of each diagonal; CSR csr_r_ptr /
// csr_c_idx / csr_diag_ptr; the FP32 values of A placed into the pattern with
// zeros at fill positions.
//
// fill_in (symbolic.cc:11-53) computes, for column i, the closure
//     S_i = A(:,i)  U  { Lpat(k) : k in S_i, k < i }     (+ the diagonal i)
// by merging sorted lists, which is quadratic in the column length.  The
// closure is the set of nodes reachable from A(:,i) in the graph whose edges
// go from every k < i to the rows of L(:,k); the same set is found here by a
// depth-first search over L with symmetric pruning (Eisenstat & Liu, "Exploiting
// structural symmetry in sparse unsymmetric symbolic factorization", SIMAX
// 1992): once U(k,i) != 0 and L(i,k) != 0, the rows of L(:,k) below i are
// reachable through i and are dropped from the search graph.  The result is the
// same set, emitted sorted, so the output is identical to the reference's.
//
// csr (symbolic.cc:55-79) is a counting-sort transpose; csr_pos additionally
// records, for every CSR entry, its position in the CSC arrays.
//
// predictLU (symbolic.cc:82-103) places A's value of row r into the LU slot of
// row r (first match in A's column order); here a per-entry slot map is built
// once (binary search in the sorted LU column) so that refactorizations only
// gather.
#include "glu_internal.h"

#include <algorithm>
#include <cstring>

namespace glu {

// Depth-first reach of column i with symmetric pruning.  Marks every reached
// node with stamp i and appends it to `found`.
static void reach_column(uint32_t i, const uint32_t *ai, uint32_t a0, uint32_t a1,
                         const std::vector<uint32_t> &sym_r_idx,
                         const std::vector<uint64_t> &lstart,  // first L row (after diag)
                         const std::vector<uint64_t> &lprune,  // pruned end of L(:,k)
                         std::vector<uint32_t> &mark, std::vector<uint32_t> &found,
                         std::vector<uint32_t> &stack_node, std::vector<uint64_t> &stack_pos) {
    for (uint32_t q = a0; q < a1; ++q) {
        uint32_t r = ai[q];
        if (mark[r] == i) continue;
        mark[r] = i;
        found.push_back(r);
        if (r >= i) continue;  // rows >= i are terminal
        // iterative DFS from r
        size_t sp = 0;
        stack_node[sp] = r;
        stack_pos[sp] = lstart[r];
        ++sp;
        while (sp > 0) {
            uint32_t k = stack_node[sp - 1];
            uint64_t p = stack_pos[sp - 1];
            uint64_t pend = lprune[k];
            bool pushed = false;
            for (; p < pend; ++p) {
                uint32_t c = sym_r_idx[p];
                if (mark[c] == i) continue;
                mark[c] = i;
                found.push_back(c);
                if (c < i) {
                    stack_pos[sp - 1] = p + 1;
                    stack_node[sp] = c;
                    stack_pos[sp] = lstart[c];
                    ++sp;
                    pushed = true;
                    break;
                }
            }
            if (!pushed) --sp;
        }
    }
}

Status symbolic_analyze(uint32_t n, uint32_t nnz_a, const uint32_t *ap, const uint32_t *ai,
                        SymbolicData &s) {
    if (n == 0) return set_error(GLU_ERR_ARG, "n must be positive");
    if (ap[0] != 0 || ap[n] != nnz_a) return set_error(GLU_ERR_ARG, "inconsistent column pointers");
    for (uint32_t i = 0; i < n; ++i)
        if (ap[i] > ap[i + 1]) return set_error(GLU_ERR_ARG, "column pointers not monotone");
    for (uint32_t q = 0; q < nnz_a; ++q)
        if (ai[q] >= n) return set_error(GLU_ERR_ARG, "row index out of range");

    s.n = n;
    s.sym_c_ptr.assign(1, 0);
    s.sym_r_idx.clear();
    s.l_col_ptr.clear();
    s.sym_c_ptr.reserve(n + 1);
    s.l_col_ptr.reserve(n);
    s.sym_r_idx.reserve(size_t(nnz_a) * 4);

    std::vector<uint64_t> lstart(n), lprune(n);
    std::vector<uint32_t> mark(n, UINT32_MAX);
    std::vector<uint32_t> found;
    found.reserve(1024);
    std::vector<uint32_t> stack_node(n + 1);
    std::vector<uint64_t> stack_pos(n + 1);
    std::vector<uint64_t> bits((n + 63) / 64, 0);
    std::vector<uint8_t> pruned(n, 0);

    for (uint32_t i = 0; i < n; ++i) {
        found.clear();
        reach_column(i, ai, ap[i], ap[i + 1], s.sym_r_idx, lstart, lprune, mark, found,
                     stack_node, stack_pos);
        if (mark[i] != i) {  // structural diagonal is always present (symbolic.cc:39-43)
            mark[i] = i;
            found.push_back(i);
        }
        // emit sorted: bitmap scan for dense columns, sort for sparse ones
        uint32_t lo = n, hi = 0;
        for (uint32_t r : found) {
            lo = std::min(lo, r);
            hi = std::max(hi, r);
        }
        size_t cnt = found.size();
        size_t span_words = (hi >> 6) - (lo >> 6) + 1;
        if (cnt > 64 && span_words < cnt * 2) {
            for (uint32_t r : found) bits[r >> 6] |= 1ull << (r & 63);
            size_t w0 = lo >> 6, w1 = hi >> 6;
            found.clear();
            for (size_t w = w0; w <= w1; ++w) {
                uint64_t b = bits[w];
                bits[w] = 0;
                while (b) {
                    int t = __builtin_ctzll(b);
                    found.push_back(uint32_t(w * 64 + t));
                    b &= b - 1;
                }
            }
        } else {
            std::sort(found.begin(), found.end());
        }
        uint64_t base = s.sym_r_idx.size();
        size_t dpos = std::lower_bound(found.begin(), found.end(), i) - found.begin();
        s.sym_r_idx.insert(s.sym_r_idx.end(), found.begin(), found.end());
        if (s.sym_r_idx.size() > UINT32_MAX)
            return set_error(GLU_ERR_NOMEM, "L+U has more than 2^32 nonzeros");
        s.l_col_ptr.push_back(uint32_t(base + dpos));
        s.sym_c_ptr.push_back(uint32_t(s.sym_r_idx.size()));
        lstart[i] = base + dpos + 1;
        lprune[i] = s.sym_r_idx.size();
        // symmetric pruning: for k in U(:,i) with L(i,k) != 0, cut L(:,k) after row i
        for (size_t t = 0; t < dpos; ++t) {
            uint32_t k = found[t];
            if (pruned[k]) continue;
            const uint32_t *b0 = s.sym_r_idx.data() + lstart[k];
            const uint32_t *b1 = s.sym_r_idx.data() + lprune[k];
            const uint32_t *hit = std::lower_bound(b0, b1, i);
            if (hit != b1 && *hit == i) {
                lprune[k] = uint64_t(hit - s.sym_r_idx.data()) + 1;
                pruned[k] = 1;
            }
        }
    }
    s.nnz = uint32_t(s.sym_r_idx.size());

    // CSR transpose (symbolic.cc:55-79) with CSC positions
    s.csr_r_ptr.assign(n + 1, 0);
    for (uint32_t p = 0; p < s.nnz; ++p) s.csr_r_ptr[s.sym_r_idx[p] + 1]++;
    for (uint32_t r = 0; r < n; ++r) s.csr_r_ptr[r + 1] += s.csr_r_ptr[r];
    s.csr_c_idx.resize(s.nnz);
    s.csr_pos.resize(s.nnz);
    s.csr_diag_ptr.resize(n);
    {
        std::vector<uint32_t> fillp(s.csr_r_ptr.begin(), s.csr_r_ptr.end() - 1);
        for (uint32_t c = 0; c < n; ++c) {
            for (uint32_t p = s.sym_c_ptr[c]; p < s.sym_c_ptr[c + 1]; ++p) {
                uint32_t r = s.sym_r_idx[p];
                uint32_t e = fillp[r]++;
                s.csr_c_idx[e] = c;
                s.csr_pos[e] = p;
                if (r == c) s.csr_diag_ptr[r] = e;
            }
        }
    }

    // slot map for value placement (predictLU semantics: first match wins)
    s.nnz_a = nnz_a;
    s.a_ptr.assign(ap, ap + n + 1);
    s.a_idx.assign(ai, ai + nnz_a);
    s.a_slot.assign(nnz_a, UINT32_MAX);
    s.lu_src.assign(s.nnz, -1);
    for (uint32_t c = 0; c < n; ++c) {
        const uint32_t *b0 = s.sym_r_idx.data() + s.sym_c_ptr[c];
        const uint32_t *b1 = s.sym_r_idx.data() + s.sym_c_ptr[c + 1];
        for (uint32_t q = ap[c]; q < ap[c + 1]; ++q) {
            const uint32_t *hit = std::lower_bound(b0, b1, ai[q]);
            uint32_t p = uint32_t(hit - s.sym_r_idx.data());
            s.a_slot[q] = p;
            if (s.lu_src[p] < 0) s.lu_src[p] = int64_t(q);
        }
    }
    return GLU_OK;
}

// predictLU: FP32 LU values from FP64 A values (zeros at fill positions).
void predict_lu(const SymbolicData &s, const double *ax, float *val) {
    for (uint32_t p = 0; p < s.nnz; ++p) {
        int64_t q = s.lu_src[p];
        val[p] = q < 0 ? 0.0f : static_cast<float>(ax[q]);
    }
}

}  // namespace glu
