/*
 * Drop-in for the reference's column loop inside MSPAI's own classes.
 *
 * Include after the reference's "Matrix.h", "Pattern.h" and "Index_Set.h"
 * (its types are used as they are) and call
 *
 *     mspai_b200_shim::Spai_GPU_Algorithm(A_sys, M_REAL, B_REAL, P, UP, epsilon_param,
 *                                         maxnew_param_local, max_impr_steps_local,
 *                                         hash_param, use_mean, pre_k_param, pre_max_param,
 *                                         count, verbose, &extra);
 *
 * in place of alg_ptr->SPAI_Algorithm(...) (src/imspai.cpp:831-833; the
 * method is non-virtual, src/Spai.h:89, so the seam is this one call).  The
 * arguments keep their meaning (src/Spai.imp:33-47); `extra` carries the
 * options that the reference passes to the algorithm object instead (-cs,
 * -ch, -qr: Switch_Algorithm::Get_Algorithm, src/Switch_Algorithm.imp:50-122)
 * and this library's own (precision, refinement, device); NULL takes the
 * library's defaults.  M is allocated as SPAI_Algorithm does on its first
 * call (count == 0: Init_Preconditioner, src/Spai.imp:68-69) and filled like
 * Com_Server::Insert_Row_Solution (src/Com_Server.cpp:416-453): per column its
 * length, row indices and values.
 *
 * The target: the reference's column routines solve for e_k and do not read
 * B (Spai_Unrestrained::SPAI_Column, src/Spai_Unrestrained.imp:78-132; only
 * Spai_Caching's Create_bk_Hat does, src/Spai_Sub.imp:735-775), so B is
 * passed on only with use_target = true (the MSPAI target [I; rho Be]).
 *
 * One MPI rank, scalar columns (A->block_size == 1; block setups go through
 * mspai_setup with bs).  Errors throw std::runtime_error with the library's
 * message, as the reference throws its own.
 */
#ifndef MSPAI_B200_REFERENCE_SHIM_HPP
#define MSPAI_B200_REFERENCE_SHIM_HPP

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "mspai_b200.h"

namespace mspai_b200_shim {

// Column c of a reference matrix (one rank: local index c) as sorted
// (row, value) runs appended to CSC arrays.
template <class Mat>
inline void append_columns(const Mat* A, int ncols, std::vector<int64_t>& ptr,
                           std::vector<int32_t>& idx, std::vector<double>& val)
{
    ptr.assign(static_cast<size_t>(ncols) + 1, 0);
    std::vector<std::pair<int32_t, double>> col;
    for (int c = 0; c < ncols; c++) {
        const int len = A->c_lines->len_cols[c];
        col.resize(len);
        for (int i = 0; i < len; i++)
            col[i] = {A->c_lines->col_idcs[c][i], A->c_lines->A[c][i]};
        std::sort(col.begin(), col.end(),
                  [](const std::pair<int32_t, double>& a, const std::pair<int32_t, double>& b) {
                      return a.first < b.first;
                  });
        for (const auto& e : col) {
            idx.push_back(e.first);
            val.push_back(e.second);
        }
        ptr[c + 1] = static_cast<int64_t>(idx.size());
    }
}

// A reference pattern (Index_Set per column) as a CSC pattern, rows sorted.
template <class Pat>
inline void pattern_columns(const Pat* P, int ncols, std::vector<int64_t>& ptr,
                            std::vector<int32_t>& idx)
{
    ptr.assign(static_cast<size_t>(ncols) + 1, 0);
    for (int c = 0; c < ncols; c++) {
        const int len = P->j_sets[c]->len;
        const size_t at = idx.size();
        idx.insert(idx.end(), P->j_sets[c]->idcs, P->j_sets[c]->idcs + len);
        std::sort(idx.begin() + at, idx.end());
        ptr[c + 1] = static_cast<int64_t>(idx.size());
    }
}

template <class Mat, class Pat>
inline void Spai_GPU_Algorithm(Mat* A, Mat*& M, Mat* B, Pat* P, Pat* UP, double epsilon_param,
                               int maxnew_param, int max_impr_steps, int hash_param,
                               const int use_mean, int pre_k_param, const int pre_max_param,
                               const int& count, const int& verbose,
                               const mspai_params* extra = nullptr, int device = 0,
                               bool use_target = false)
{
    (void)hash_param;    // remote-column hash table: one rank holds C whole
    (void)pre_k_param;   // prefetching: likewise
    (void)pre_max_param;
    if (A->block_size != 1)
        throw std::runtime_error("Spai_GPU_Algorithm: scalar columns only (block setups: "
                                 "mspai_setup with bs)");
    const int n = A->n;
    if (A->my_nbr_cols != n)
        throw std::runtime_error("Spai_GPU_Algorithm: one MPI rank holds every column");
    if (count == 0)
        A->Init_Preconditioner(M, A->n, P->len, P, maxnew_param, max_impr_steps);

    std::vector<int64_t> cptr, bptr, pptr, uptr;
    std::vector<int32_t> cidx, bidx, pidx, uidx;
    std::vector<double> cval, bval;
    append_columns(A, n, cptr, cidx, cval);
    pattern_columns(P, n, pptr, pidx);
    mspai_csc C{A->m, n, cptr[n], cptr.data(), cidx.data(), cval.data(), MSPAI_MEM_HOST};
    mspai_csc Pm{n, n, pptr[n], pptr.data(), pidx.data(), nullptr, MSPAI_MEM_HOST};
    mspai_csc Bm{}, Um{};
    if (!use_target)
        B = nullptr;
    if (B) {
        append_columns(B, n, bptr, bidx, bval);
        Bm = mspai_csc{B->m, n, bptr[n], bptr.data(), bidx.data(), bval.data(), MSPAI_MEM_HOST};
    }
    if (UP) {
        pattern_columns(UP, n, uptr, uidx);
        Um = mspai_csc{n, n, uptr[n], uptr.data(), uidx.data(), nullptr, MSPAI_MEM_HOST};
    }

    mspai_params prm;
    if (extra)
        prm = *extra;
    else
        mspai_default_params(&prm);
    prm.ep = epsilon_param;
    prm.mn = maxnew_param;
    prm.ns = max_impr_steps;
    prm.um = use_mean;
    prm.bs = 1;
    prm.probing = A->m > n ? 1 : 0;  // probing rows below A's n rows
    prm.verbose = verbose;

    mspai_handle* h = nullptr;
    if (mspai_create(&h, device, nullptr) != MSPAI_OK)
        throw std::runtime_error("Spai_GPU_Algorithm: no CUDA device");
    if (mspai_setup(h, &C, nullptr, B ? &Bm : nullptr, &Pm, UP ? &Um : nullptr, &prm) !=
        MSPAI_OK) {
        const std::string msg = mspai_last_error(h);
        mspai_free(h);
        throw std::runtime_error(msg);
    }
    int64_t nnz = 0;
    mspai_result_nnz(h, &nnz);
    std::vector<int64_t> mp(static_cast<size_t>(n) + 1);
    std::vector<int32_t> mi(static_cast<size_t>(std::max<int64_t>(nnz, 1)));
    std::vector<double> mv(static_cast<size_t>(std::max<int64_t>(nnz, 1)));
    const int rc = mspai_result_copy(h, mp.data(), mi.data(), mv.data(), MSPAI_MEM_HOST);
    mspai_free(h);
    if (rc != MSPAI_OK)
        throw std::runtime_error("Spai_GPU_Algorithm: the result could not be read");
    // Insert_Row_Solution for every column: its capacity is
    // max_block_size^2 (P->max_nnz + maxnew * nbsteps), |J_k| never exceeds it
    for (int c = 0; c < n; c++) {
        const int len = static_cast<int>(mp[c + 1] - mp[c]);
        M->c_lines->len_cols[c] = len;
        std::copy(mi.begin() + mp[c], mi.begin() + mp[c + 1], M->c_lines->col_idcs[c]);
        std::copy(mv.begin() + mp[c], mv.begin() + mp[c + 1], M->c_lines->A[c]);
    }
}

}  // namespace mspai_b200_shim

#endif
