/*
 * CPU restatement of the MSPAI column loop -- TEST INFRASTRUCTURE ONLY.
 *
 * This is the oracle the GPU product is checked against.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it; the
 * product never calls it.
 *
 * It restates, per column k, the reference's Spai_Unrestrained::SPAI_Column
 * (src/Spai_Unrestrained.imp:33-133) and its block variant
 * (src/Spai_Unrestrained_Block.imp:33-140) with the same dense LAPACK calls
 * (dgeqrf / dormqr / dtrtrs / dgemv / dgemm, src/Spai_Sub.cpp:46-174) and the
 * same std::sort calls, so that on the same inputs it reproduces the
 * reference's results to the last bit where the reference is deterministic.
 * The right-hand side is B(I,k) merged as in Spai_Sub::Create_bk_Hat
 * (src/Spai_Sub.imp:735-775) when a target B is given (the reference's
 * B-aware Spai_Caching path, src/Spai_Caching.imp:115-118), else e_k as in
 * Create_ek_Hat (src/Spai_Sub.imp:629-658).
 *
 * LAPACK is the one bundled with scipy, reached through oracle/ref_shim's
 * forwarding layer (the same one the compiled reference uses).
 */
#include "ref_shim/mkl.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

struct Csc {
    int nrows, ncols;
    const int64_t* ptr;
    const int32_t* idx;
    const double* val;  // may be null for a pattern
};

struct RhoIdx {  // RHO_IDX, src/Matrix.h:135-138
    int idx;
    double rho;
};
struct RhoLess {  // RHO_Comparator, src/Matrix.h:145-150
    bool operator()(const RhoIdx& a, const RhoIdx& b) const { return a.rho < b.rho; }
};

// Spai_Sub::Get_I_Set (src/Spai_Sub.imp:65-122): union of the row indices of
// the columns in J, then std::sort.  Block size 1.
void get_i_set(const Csc& C, const std::vector<int>& J, std::vector<char>& mark,
               std::vector<int>& I)
{
    I.clear();
    for (int j : J)
        for (int64_t p = C.ptr[j]; p < C.ptr[j + 1]; p++) {
            int r = C.idx[p];
            if (!mark[r]) {
                mark[r] = 1;
                I.push_back(r);
            }
        }
    std::sort(I.begin(), I.end());
    for (int r : I)
        mark[r] = 0;
}

// Spai_Sub::Create_Submatrix_AHat (src/Spai_Sub.imp:221-282): dense C(I,J),
// column-major, ld = |I|, via a merge of each column against I.
void create_ahat(const Csc& C, const std::vector<int>& J, const std::vector<int>& I,
                 std::vector<double>& Ahat)
{
    const size_t m = I.size(), n = J.size();
    Ahat.assign(m * n, 0.0);
    for (size_t jj = 0; jj < n; jj++) {
        const int j = J[jj];
        int64_t p = C.ptr[j];
        const int64_t pe = C.ptr[j + 1];
        for (size_t i = 0; i < m && p < pe; i++)
            if (I[i] == C.idx[p]) {
                Ahat[jj * m + i] = C.val[p];
                p++;
            }
    }
}

// Right-hand side: Create_bk_Hat(A,M,B,...) (src/Spai_Sub.imp:735-775) when B
// is given, else Create_ek_Hat (src/Spai_Sub.imp:629-658).
void create_rhs(const Csc* B, const std::vector<int>& I, int col, std::vector<double>& b)
{
    const size_t m = I.size();
    b.assign(m, 0.0);
    if (B) {
        int64_t p = B->ptr[col];
        const int64_t pe = B->ptr[col + 1];
        size_t q = 0;
        while (p < pe && q < m) {
            const int ib = B->idx[p], ii = I[q];
            if (ib < ii)
                p++;
            else if (ib > ii)
                q++;
            else {
                b[q] = B->val[p];
                p++;
                q++;
            }
        }
    }
    else {
        for (size_t i = 0; i < m; i++) {
            if (I[i] > col)
                break;
            if (I[i] == col) {
                b[i] = 1.0;
                break;
            }
        }
    }
}

// Spai_Unrestrained::Approximative_Solution (src/Spai_Unrestrained.imp:135-195):
// dgeqrf, dormqr(L,T), compaction of R (Ectract_Quadratic_Content,
// src/Spai_Sub.imp:585-601), dtrtrs(U,N,N).  nrhs = 1 (scalar) or bs (block).
// x: m x nrhs (ld m) on entry, solution in its first n rows (ld m) on exit.
int ls_solve(std::vector<double> A, int m, int n, int nrhs, double* x, int ldx)
{
    int info = 0, lwork = -1;
    const int lda = std::max(m, 1);
    const int k = std::min(m, n);
    std::vector<double> tau(std::max(k, 1));
    double wq = 0.0;
    dgeqrf(&m, &n, A.data(), &lda, tau.data(), &wq, &lwork, &info);
    lwork = std::max(1, static_cast<int>(wq));
    std::vector<double> work(lwork);
    dgeqrf(&m, &n, A.data(), &lda, tau.data(), work.data(), &lwork, &info);
    lwork = -1;
    dormqr("L", "T", &m, &nrhs, &k, A.data(), &lda, tau.data(), x, &ldx, &wq, &lwork, &info);
    lwork = std::max(1, static_cast<int>(wq));
    work.assign(lwork, 0.0);
    dormqr("L", "T", &m, &nrhs, &k, A.data(), &lda, tau.data(), x, &ldx, work.data(), &lwork,
           &info);
    // compact the leading n x n upper triangle to ld = n
    if (m > n)
        for (int c = 0; c < n; c++)
            std::memmove(&A[static_cast<size_t>(c) * n], &A[static_cast<size_t>(c) * m],
                         n * sizeof(double));
    const int ldr = std::max(1, n);
    int tinfo = 0;
    dtrtrs("U", "N", "N", &n, &nrhs, A.data(), &ldr, x, &ldx, &tinfo);
    return tinfo;
}

}  // namespace

extern "C" {

/*
 * Scalar SPAI / MSPAI setup for columns [col_lo, col_hi), or, when col_list
 * is not null, for the columns col_list[col_lo .. col_hi).
 *
 * C      : nrows x n CSC (rows >= n are probing rows), sorted rows.
 * Crow   : CSR row structure of C's first n rows (column indices per row,
 *          sorted), used for candidates (Union_Nl_Sets, src/Spai_Sub.imp:124-200);
 *          may be null when ns == 0.
 * B      : target CSC (nullable; null means e_k, the Spai_Unrestrained path).
 * P, UP  : start pattern and optional upper pattern (CSC pattern).
 * Output : for column k, out_len[k] entries written at out_idx/out_val +
 *          k * out_stride (sorted J and m_k), out_res[k] = ||C(I,J) m - b||_2,
 *          out_steps[k] = number of LS solves, out_info[k] = dtrtrs info.
 */
int oracle_spai_scalar(int nrows, int n, const int64_t* cptr, const int32_t* cidx,
                       const double* cval, const int64_t* rptr, const int32_t* rcol,
                       const int64_t* bptr, const int32_t* bidx, const double* bval,
                       const int64_t* pptr, const int32_t* pidx, const int64_t* upptr,
                       const int32_t* upidx, double ep, int mn, int ns, int um, int col_lo,
                       int col_hi, int out_stride, int32_t* out_len, int32_t* out_idx,
                       double* out_val, double* out_res, int32_t* out_steps, int32_t* out_info,
                       const int32_t* col_list)
{
    Csc C{nrows, n, cptr, cidx, cval};
    Csc Bm{nrows, n, bptr, bidx, bval};
    const Csc* B = bptr ? &Bm : nullptr;
    std::vector<char> mark(std::max(nrows, n) + 1, 0);
    std::vector<int> J, I, L, U, Jt;
    std::vector<double> Ahat, b, bk, r;
    std::vector<RhoIdx> rhos;

    for (int it = col_lo; it < col_hi; it++) {
        const int col = col_list ? col_list[it] : it;
        // Com_Server::Get_P_Col (src/Com_Server.imp:446-470)
        J.assign(pidx + pptr[col], pidx + pptr[col + 1]);
        double res = 1.0e50;
        int steps = 0, info = 0;
        std::vector<double> x;
        for (int step = -1; step < ns; step++) {  // src/Spai_Unrestrained.imp:78
            get_i_set(C, J, mark, I);
            create_ahat(C, J, I, Ahat);
            const int m = static_cast<int>(I.size());
            const int nn = static_cast<int>(J.size());
            create_rhs(B, I, col, b);
            bk = b;
            x = b;
            x.resize(std::max<size_t>(x.size(), J.size()), 0.0);
            info = ls_solve(Ahat, m, nn, 1, x.data(), std::max(m, 1));
            steps++;
            // Spai_Sub::Residual_Norm (src/Spai_Sub.imp:915-941): r = Ahat m - b
            {
                const char* T = "N";
                int lda = std::max(m, 1), inc = 1;
                double alpha = 1.0, beta = -1.0;
                r = bk;
                if (m > 0 && nn > 0)
                    dgemv(T, &m, &nn, &alpha, Ahat.data(), &lda, x.data(), &inc, &beta,
                          r.data(), &inc);
                else
                    for (auto& v : r)
                        v = -v;
                double s = 0.0;
                for (int i = 0; i < m; i++)
                    s += r[i] * r[i];
                res = std::sqrt(s);
            }
            if (res <= ep || step == ns - 1)  // src/Spai_Unrestrained.imp:118-121
                break;

            // Spai_Sub::Augment_Sparsity (src/Spai_Sub.imp:1010-1116)
            L = I;
            if (std::find(I.begin(), I.end(), col) == I.end())
                L.push_back(col);
            U.clear();
            for (int l : L) {  // Union_Nl_Sets, non-symmetric branch
                for (int64_t p = rptr[l]; p < rptr[l + 1]; p++) {
                    int c = rcol[p];
                    if (!mark[c]) {
                        mark[c] = 1;
                        U.push_back(c);
                    }
                }
            }
            for (int c : U)
                mark[c] = 0;
            std::sort(U.begin(), U.end());
            Jt.resize(U.size());
            Jt.erase(std::set_difference(U.begin(), U.end(), J.begin(), J.end(), Jt.begin()),
                     Jt.end());
            if (upptr) {  // Index_Set::Set_Intersection with UP(:,col)
                std::vector<int> T;
                std::set_intersection(Jt.begin(), Jt.end(), upidx + upptr[col],
                                      upidx + upptr[col + 1], std::back_inserter(T));
                Jt.swap(T);
            }
            if (Jt.empty())
                break;
            // Spai_Sub::Compute_Rhos (src/Spai_Sub.imp:1231-1348) and
            // Compute_Numerator (src/Spai_Sub.cpp:252-291)
            rhos.resize(Jt.size());
            double mean = 0.0;
            for (size_t t = 0; t < Jt.size(); t++) {
                const int j = Jt[t];
                double s2 = 0.0;
                for (int64_t p = cptr[j]; p < cptr[j + 1]; p++)
                    s2 += cval[p] * cval[p];
                const double ajn = std::sqrt(s2);
                double num = 0.0;
                for (int64_t p = cptr[j]; p < cptr[j + 1]; p++) {
                    const int ri = cidx[p];
                    for (int q = 0; q < m; q++) {
                        if (ri < I[q])
                            break;
                        if (I[q] == ri)
                            num += r[q] * cval[p];
                    }
                }
                num *= num;
                double rho = res * res - num / (ajn * ajn);
                rho = std::sqrt(rho);
                mean += rho;
                rhos[t].idx = j;
                rhos[t].rho = rho;
            }
            if (um)
                mean /= static_cast<double>(Jt.size());
            std::sort(rhos.begin(), rhos.end(), RhoLess());
            for (int el = 0; el < mn && el < static_cast<int>(Jt.size()) && rhos[el].rho <= mean;
                 el++)
                J.push_back(rhos[el].idx);
            std::sort(J.begin(), J.end());
        }
        // Insert_Row_Solution (src/Spai_Sub.imp:603-627)
        const int nn = static_cast<int>(J.size());
        out_len[col] = nn;
        if (nn > out_stride)
            return -1 - col;
        for (int i = 0; i < nn; i++) {
            out_idx[static_cast<size_t>(col) * out_stride + i] = J[i];
            out_val[static_cast<size_t>(col) * out_stride + i] = x[i];
        }
        out_res[col] = res;
        out_steps[col] = steps;
        out_info[col] = info;
    }
    return 0;
}


/*
 * Block SPAI with a constant block size bs (Spai_Unrestrained_Block::
 * SPAI_Column, src/Spai_Unrestrained_Block.imp:33-140), restated on the
 * scalar CSC of C:
 *   - block column kb has the scalar columns bs*kb .. bs*kb+bs-1; the block
 *     pattern Pb gives J (block indices); I is the set of block rows that the
 *     blocks of C(:, J) touch (rows >= n_s, probing rows, are single rows);
 *   - A_hat = C(I, J) expanded to scalars (Create_Submatrix_AHat_Block,
 *     src/Spai_Sub.imp:284-401), the right-hand side is the identity block at
 *     block row kb (Create_ek_Hat_Block, :690-733) or B(I, bs*kb + c);
 *   - dgeqrf / dormqr / dtrtrs with nrhs = bs (src/Spai_Unrestrained_Block.imp:
 *     142-205), residual R = A_hat X - E and its Frobenius norm
 *     (Residual_Norm_Block, src/Spai_Sub.imp:943-975), stop at ep * sqrt(bs);
 *   - pattern update (Augment_Sparsity_Block, src/Spai_Sub.imp:1118-1229):
 *     candidates are the block columns of the block rows of L = I u {kb},
 *     rho_j^2 = ||R||_F^2 - <N, (A_j^T A_j)^-1 N> with N = A_j(I)^T R
 *     (Compute_Rhos_Block :1350-1465, Compute_Numerator_Block
 *     src/Spai_Sub.cpp:293-367; the inverse by dgetrf/dgetri as
 *     Compute_Square_Inverse, src/Matrix.imp:2945-3030).
 * Output: scalar column bs*kb + c of M holds rows expanded(J) and X(:, c).
 */
int oracle_spai_block(int nrows, int n_s, int bs, const int64_t* cptr, const int32_t* cidx,
                      const double* cval, const int64_t* rptr, const int32_t* rcol,
                      const int64_t* bptr, const int32_t* bidx, const double* bval,
                      const int64_t* pbptr, const int32_t* pbidx, double ep, int mn, int ns,
                      int um, int kb_lo, int kb_hi, int out_stride, int32_t* out_len,
                      int32_t* out_idx, double* out_val, double* out_res, int32_t* out_steps,
                      int32_t* out_info, const int32_t* blk_list)
{
    const int nb = n_s / bs;
    if (nb * bs != n_s)
        return -1000000;
    const int nblocks_rows = nb + (nrows - n_s);  // probing rows are blocks of one
    auto row_block = [&](int r) { return r < n_s ? r / bs : nb + (r - n_s); };
    auto block_first = [&](int b) { return b < nb ? b * bs : n_s + (b - nb); };
    auto block_height = [&](int b) { return b < nb ? bs : 1; };
    std::vector<char> mark(std::max(nblocks_rows, nb) + 1, 0);
    std::vector<int> J, I, L, U, Jt, rowoff;
    std::vector<double> Ahat, E, X, R;
    std::vector<RhoIdx> rhos;
    for (int it = kb_lo; it < kb_hi; it++) {
        const int kb = blk_list ? blk_list[it] : it;  // block columns [lo, hi) or a list
        J.assign(pbidx + pbptr[kb], pbidx + pbptr[kb + 1]);
        double res = 1.0e50;
        int steps = 0, info = 0;
        const double ep_eff = ep * std::sqrt(static_cast<double>(bs));
        int m = 0, n = 0;
        for (int step = -1; step < ns; step++) {
            // I: block rows touched by C(:, J)
            I.clear();
            for (int jb : J)
                for (int c = jb * bs; c < jb * bs + bs; c++)
                    for (int64_t p = cptr[c]; p < cptr[c + 1]; p++) {
                        const int b = row_block(cidx[p]);
                        if (!mark[b]) {
                            mark[b] = 1;
                            I.push_back(b);
                        }
                    }
            std::sort(I.begin(), I.end());
            for (int b : I)
                mark[b] = 0;
            rowoff.assign(I.size() + 1, 0);
            for (size_t i = 0; i < I.size(); i++)
                rowoff[i + 1] = rowoff[i] + block_height(I[i]);
            m = rowoff[I.size()];
            n = static_cast<int>(J.size()) * bs;
            // A_hat (m x n, column-major): scatter each scalar column
            Ahat.assign(static_cast<size_t>(m) * n, 0.0);
            for (size_t jj = 0; jj < J.size(); jj++)
                for (int a = 0; a < bs; a++) {
                    const int c = J[jj] * bs + a;
                    for (int64_t p = cptr[c]; p < cptr[c + 1]; p++) {
                        const int r = cidx[p];
                        const int b = row_block(r);
                        const size_t q = std::lower_bound(I.begin(), I.end(), b) - I.begin();
                        const int row = rowoff[q] + (r - block_first(b));
                        Ahat[(jj * bs + a) * static_cast<size_t>(m) + row] = cval[p];
                    }
                }
            // right-hand side E (m x bs)
            E.assign(static_cast<size_t>(m) * bs, 0.0);
            for (int cc = 0; cc < bs; cc++) {
                const int col = kb * bs + cc;
                if (bptr) {
                    for (int64_t p = bptr[col]; p < bptr[col + 1]; p++) {
                        const int r = bidx[p];
                        const int b = row_block(r);
                        const auto it = std::lower_bound(I.begin(), I.end(), b);
                        if (it != I.end() && *it == b)
                            E[cc * static_cast<size_t>(m) + rowoff[it - I.begin()] +
                              (r - block_first(b))] = bval[p];
                    }
                }
                else {
                    const auto it = std::lower_bound(I.begin(), I.end(), kb);
                    if (it != I.end() && *it == kb)
                        E[cc * static_cast<size_t>(m) + rowoff[it - I.begin()] + cc] = 1.0;
                }
            }
            X = E;
            X.resize(std::max<size_t>(X.size(), static_cast<size_t>(n) * bs), 0.0);
            info = ls_solve(Ahat, m, n, bs, X.data(), std::max(m, 1));
            steps++;
            // R = A_hat X - E (X's first n rows, ld m)
            R = E;
            {
                const char* T = "N";
                int lda = std::max(m, 1), ldb = std::max(m, 1), ldc = std::max(m, 1), nr = bs;
                double alpha = 1.0, beta = -1.0;
                if (m > 0 && n > 0)
                    dgemm(T, T, &m, &nr, &n, &alpha, Ahat.data(), &lda, X.data(), &ldb, &beta,
                          R.data(), &ldc);
                else
                    for (auto& v : R)
                        v = -v;
            }
            double s2 = 0.0;
            for (double v : R)
                s2 += v * v;
            res = std::sqrt(s2);
            if (res <= ep_eff || step == ns - 1)
                break;
            // candidates: block columns of the block rows of L = I u {kb}
            L.clear();
            for (int b : I)
                if (b < nb)
                    L.push_back(b);
            if (std::find(L.begin(), L.end(), kb) == L.end())
                L.push_back(kb);
            U.clear();
            for (int l : L)
                for (int r = l * bs; r < l * bs + bs; r++)
                    for (int64_t p = rptr[r]; p < rptr[r + 1]; p++) {
                        const int cb = rcol[p] / bs;
                        if (!mark[cb]) {
                            mark[cb] = 1;
                            U.push_back(cb);
                        }
                    }
            for (int c : U)
                mark[c] = 0;
            std::sort(U.begin(), U.end());
            Jt.resize(U.size());
            Jt.erase(std::set_difference(U.begin(), U.end(), J.begin(), J.end(), Jt.begin()),
                     Jt.end());
            if (Jt.empty())
                break;
            rhos.resize(Jt.size());
            double mean = 0.0;
            for (size_t t = 0; t < Jt.size(); t++) {
                const int jb = Jt[t];
                // N = A_j(I)^T R (bs x bs), G = A_j^T A_j (bs x bs, whole column)
                std::vector<double> N(static_cast<size_t>(bs) * bs, 0.0), G(N.size(), 0.0);
                for (int a = 0; a < bs; a++) {
                    const int c = jb * bs + a;
                    for (int64_t p = cptr[c]; p < cptr[c + 1]; p++) {
                        const int r = cidx[p];
                        const int b = row_block(r);
                        const auto it = std::lower_bound(I.begin(), I.end(), b);
                        if (it == I.end() || *it != b)
                            continue;
                        const int row = rowoff[it - I.begin()] + (r - block_first(b));
                        for (int q = 0; q < bs; q++)
                            N[a + q * bs] += cval[p] * R[q * static_cast<size_t>(m) + row];
                    }
                    for (int a2 = 0; a2 < bs; a2++) {
                        const int c2 = jb * bs + a2;
                        int64_t p = cptr[c], q = cptr[c2];
                        double g = 0.0;
                        while (p < cptr[c + 1] && q < cptr[c2 + 1]) {
                            if (cidx[p] < cidx[q])
                                p++;
                            else if (cidx[p] > cidx[q])
                                q++;
                            else
                                g += cval[p++] * cval[q++];
                        }
                        G[a + a2 * bs] = g;
                    }
                }
                // G^-1 via dgetrf/dgetri (Compute_Square_Inverse)
                {
                    int nn = bs, lda = bs, inf = 0, lw = -1;
                    std::vector<int> ipiv(bs);
                    dgetrf_(&nn, &nn, G.data(), &lda, ipiv.data(), &inf);
                    double wq = 0.0;
                    dgetri_(&nn, G.data(), &lda, ipiv.data(), &wq, &lw, &inf);
                    lw = std::max(1, static_cast<int>(wq));
                    std::vector<double> wk(lw);
                    dgetri_(&nn, G.data(), &lda, ipiv.data(), wk.data(), &lw, &inf);
                }
                double term = 0.0;
                for (int q = 0; q < bs; q++)
                    for (int a = 0; a < bs; a++) {
                        double bm = 0.0;
                        for (int a2 = 0; a2 < bs; a2++)
                            bm += G[a + a2 * bs] * N[a2 + q * bs];
                        term += bm * N[a + q * bs];
                    }
                double rho = std::sqrt(res * res - term);
                mean += rho;
                rhos[t].idx = jb;
                rhos[t].rho = rho;
            }
            if (um)
                mean /= static_cast<double>(Jt.size());
            std::sort(rhos.begin(), rhos.end(), RhoLess());
            for (int el = 0; el < mn && el < static_cast<int>(Jt.size()) && rhos[el].rho <= mean;
                 el++)
                J.push_back(rhos[el].idx);
            std::sort(J.begin(), J.end());
        }
        // scalar columns of block column kb
        const int len = static_cast<int>(J.size()) * bs;
        for (int cc = 0; cc < bs; cc++) {
            const int col = kb * bs + cc;
            out_len[col] = len;
            if (len > out_stride)
                return -1 - col;
            for (int jj = 0; jj < len; jj++) {
                out_idx[static_cast<size_t>(col) * out_stride + jj] = J[jj / bs] * bs + jj % bs;
                out_val[static_cast<size_t>(col) * out_stride + jj] =
                    X[cc * static_cast<size_t>(m) + jj];
            }
            out_res[col] = res;
            out_steps[col] = steps;
            out_info[col] = info;
        }
    }
    return 0;
}

}  // extern "C"
