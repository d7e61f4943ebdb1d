/*
 * Serial driver for the reference MSPAI sources, compiled here from the files
 * where they lie (see oracle/Makefile).  TEST INFRASTRUCTURE: it is the
 * checker and the CPU baseline, never part of the product.
 *
 * It follows the upstream serial command line
 *     mspai <A.mtx> <pattern.mtx|-1|-2> <B.mtx|-1> [options]
 * (reference doc/mspai-1.2.pdf section 2.2; -1 = diagonal start pattern,
 * -2 = pattern of C, target -1 = identity) and the setup sequence of
 * PC_MSPAI::bspai (src/imspai.cpp:648-924) with the Matrix Market readers in
 * place of the PETSc conversion:
 *   Read_mm_Matrix::Read_Matrix_File   (src/Read_mm_Matrix.cpp:115-231)
 *   Matrix::Convert_Block_Matrix        (src/Matrix.imp:1280) when -bs != 1
 *   Read_mm_Matrix::Read_Target_File    (src/Read_mm_Matrix.cpp:233-420)
 *   Pattern_Switch::Generate_Pattern    (src/Pattern_Switch.cpp:35-94)
 *   Switch_Algorithm::Get_Algorithm     (src/Switch_Algorithm.imp:37-122)
 *   Spai::SPAI_Algorithm                (src/Spai.imp:33-191)
 *   Matrix::Write_Matrix_To_File        (src/Matrix.cpp:251-340)
 *
 * Two departures, both outside the reference sources:
 *  - Data_To_Matrix leaves block_size / block_sizes unset
 *    (src/Read_mm_Matrix.cpp:669-845); they are set to 1 here as the PETSc
 *    path does (src/Matrix.imp:910-914).
 *  - Init_Preconditioner sizes its per-column work buffers for at most 10000
 *    index entries, 40000 values of A(I,J) and 1000 LAPACK work entries
 *    (src/Matrix.imp:185-188, 245-263), which overflow on large columns.  The
 *    driver calls Init_Preconditioner itself, replaces those buffers with ones
 *    sized from the actual problem, and then runs SPAI_Algorithm with count=1
 *    so it does not re-initialise them (src/Spai.imp:67-81).  Nothing else
 *    depends on count for the no_opt / caching / qr_updates algorithms.
 *
 * Extra driver options (not in the reference):
 *   -cols a:b   run SPAI_Column for columns [a, b) only (timed subset)
 *   -colfile f  run SPAI_Column for the (block) columns listed in f, one index
 *               per line (a stratified sample of a large problem)
 *   -repeat r   with a column subset: run the column loop r times after one
 *               read of the inputs (each pass recomputes the same columns)
 *   -time f     write {"setup_s":…, "columns":…, "rep_s": [...]} as JSON to f
 *   -gpu fp64|mixed   (ref_driver_gpu only, built with MSPAI_GPU_SHIM) run the
 *               library's drop-in mspai_b200_shim::Spai_GPU_Algorithm
 *               (include/mspai_b200_reference_shim.hpp) in place of
 *               alg->SPAI_Algorithm, as a maintainer would in
 *               PC_MSPAI::bspai, and write M with the reference's own
 *               Write_Matrix_To_File: the stock and the drop-in runs of one
 *               command line give files that the tests compare
 * With a subset, only the computed columns are written (scalar columns; a
 * block column as its bs scalar columns, through the reference's
 * Matrix::Scalar_Matrix).
 */
#include "Matrix.h"
#include "Pattern.h"
#include "Pattern_Switch.h"
#include "Read_mm_Matrix.h"
#include "Spai.h"
#include "Switch_Algorithm.h"

#ifdef MSPAI_GPU_SHIM
#include "mspai_b200_reference_shim.hpp"
#endif

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

struct Options {
    const char* a_file = nullptr;
    const char* p_file = nullptr;  // nullptr when pp = 1 or 2
    const char* b_file = nullptr;  // nullptr when tp = 1
    int pp = 1, tp = 1;
    const char* up_file = nullptr;
    int up = 3;
    double ep = 0.4;
    int mn = 5, ns = 5, hs = 6, cs = 0, qr = 0, ch = 0, pk = 0, pm = 0, us = 0;
    int um = 1, bs = 1, vb = 0;
    double fg = 0.3, rho = 1.0;
    const char* ce = nullptr;
    const char* be = nullptr;
    const char* out = "precond.mtx";
    long col_lo = -1, col_hi = -1;
    const char* col_file = nullptr;
    int repeat = 1;
    const char* time_file = nullptr;
    const char* gpu = nullptr;  // -gpu fp64|mixed: the library's drop-in
};

void usage()
{
    std::fprintf(stderr,
                 "usage: ref_driver <A.mtx> <pattern.mtx|-1|-2> <B.mtx|-1> [-ep x] [-mn k] "
                 "[-ns k] [-hs k] [-cs k] [-qr k] [-fg x] [-um 0|1] [-ch 0|1] [-Ce f] [-Be f] "
                 "[-rho x] [-schur 0|1] [-up f|1|2] [-pk k] [-pm 0|1] [-bs k] [-vb k] "
                 "[-out f] [-cols a:b] [-colfile f] [-repeat r] [-time f]\n");
    std::exit(2);
}

Options parse(int argc, char** argv)
{
    Options o;
    if (argc < 4)
        usage();
    o.a_file = argv[1];
    if (!std::strcmp(argv[2], "-1"))
        o.pp = 1;
    else if (!std::strcmp(argv[2], "-2"))
        o.pp = 2;
    else {
        o.pp = 0;
        o.p_file = argv[2];
    }
    if (!std::strcmp(argv[3], "-1"))
        o.tp = 1;
    else {
        o.tp = 0;
        o.b_file = argv[3];
    }
    for (int i = 4; i < argc; i += 2) {
        if (i + 1 >= argc)
            usage();
        const std::string k = argv[i];
        const char* v = argv[i + 1];
        if (k == "-ep") o.ep = std::atof(v);
        else if (k == "-mn") o.mn = std::atoi(v);
        else if (k == "-ns") o.ns = std::atoi(v);
        else if (k == "-hs") o.hs = std::atoi(v);
        else if (k == "-cs") o.cs = std::atoi(v);
        else if (k == "-qr") o.qr = std::atoi(v);
        else if (k == "-fg") o.fg = std::atof(v);
        else if (k == "-um") o.um = std::atoi(v);
        else if (k == "-ch") o.ch = std::atoi(v);
        else if (k == "-pk") o.pk = std::atoi(v);
        else if (k == "-pm") o.pm = std::atoi(v);
        else if (k == "-schur") o.us = std::atoi(v);
        else if (k == "-rho") o.rho = std::atof(v);
        else if (k == "-Ce") o.ce = v;
        else if (k == "-Be") o.be = v;
        else if (k == "-bs") o.bs = std::atoi(v);
        else if (k == "-vb") o.vb = std::atoi(v);
        else if (k == "-out") o.out = v;
        else if (k == "-time") o.time_file = v;
        else if (k == "-up") {
            if (!std::strcmp(v, "1")) o.up = 1;
            else if (!std::strcmp(v, "2")) o.up = 2;
            else { o.up = 0; o.up_file = v; }
        }
        else if (k == "-colfile") o.col_file = v;
        else if (k == "-gpu") o.gpu = v;
        else if (k == "-repeat") o.repeat = std::atoi(v) > 0 ? std::atoi(v) : 1;
        else if (k == "-cols") {
            if (std::sscanf(v, "%ld:%ld", &o.col_lo, &o.col_hi) != 2)
                usage();
        }
        else
            usage();
    }
    return o;
}

// Names the protected virtual Spai<double>::SPAI_Column through a derived
// class so that the driver can run the reference's per-column routine on a
// column range.
struct Column_Access : Spai<double> {
    using Column_Fn = void (Spai<double>::*)(Matrix<double>*, Matrix<double>*&, Matrix<double>*,
                                             Pattern*, Pattern*, Index_Set*, const int,
                                             const double, const int, const int,
                                             Hash_Table<double>*, const int, int, const int,
                                             unsigned int*&, unsigned int*&);
    static Column_Fn fn() { return &Column_Access::SPAI_Column; }
};

template <class T>
void replace_buffer(T*& p, size_t count)
{
    delete[] p;
    p = new T[count]();
}

}  // namespace

int main(int argc, char** argv)
{
    Options o = parse(argc, argv);
    MPI_Comm world = MPI_COMM_WORLD;
    const int hash_sizes[7] = {0, 101, 503, 2503, 12503, 62501, 104743};
    try {
        if (o.hs < 0 || o.hs > 6)
            throw std::runtime_error("illegal -hs");
        Read_mm_Matrix rm;
        Matrix<double>* A = nullptr;
        Matrix<double>* B = nullptr;
        bool symmetric = false;
        int prob_Ce_N = 0;
        const bool use_prob = o.ce != nullptr;
        rm.Read_Matrix_File(const_cast<char*>(o.a_file), const_cast<char*>(o.ce), use_prob, o.us,
                            symmetric, false, A, prob_Ce_N, o.rho, world);
        A->block_size = 1;
        A->max_block_size = 1;
        A->block_sizes = new int[A->m > A->n ? A->m : A->n];
        for (int i = 0; i < (A->m > A->n ? A->m : A->n); i++)
            A->block_sizes[i] = 1;

        Matrix<double>* A_sys = A;
        if (o.bs != 1)
            A_sys = Matrix<double>::Convert_Block_Matrix(A, o.bs, 1000000, 0);

        rm.Read_Target_File(A_sys, const_cast<char*>(o.b_file), const_cast<char*>(o.be), use_prob,
                            o.us, B, prob_Ce_N, o.tp, o.rho, o.vb, world);

        Pattern_Switch<double> ps;
        Pattern loader(0, 0, world);  // Arbitrary_Pattern is a non-static member
        Pattern* P_arb = nullptr;
        if (o.pp == 0)
            P_arb = loader.Arbitrary_Pattern(const_cast<char*>(o.p_file), A_sys->n, o.us,
                                               prob_Ce_N, world);
        Pattern* P = ps.Generate_Pattern(A_sys, nullptr, P_arb, o.pp, o.us, prob_Ce_N, use_prob,
                                         1, o.vb);
        Pattern* UP = nullptr;
        if (o.up < 3) {
            Pattern* UP_arb = nullptr;
            if (o.up == 0)
                UP_arb = loader.Arbitrary_Pattern(const_cast<char*>(o.up_file), A_sys->n, o.us,
                                                    prob_Ce_N, world);
            UP = ps.Generate_Pattern(A_sys, nullptr, UP_arb, o.up, o.us, prob_Ce_N, use_prob, 1,
                                     o.vb);
        }

        // opt_level as in src/imspai.cpp:483-491
        int opt_level = 0;
        if (o.cs > 0)
            opt_level = 1;
        if (o.ch > 0)
            opt_level = 2;
        if (o.qr > 0 && o.ns > 0 && o.mn > 0)
            opt_level = 3;
        Switch_Algorithm<double> sa;
        Spai<double>* alg = sa.Get_Algorithm(0, opt_level, o.cs, o.qr, o.fg, o.bs, o.vb);

        // Preconditioner set-up with buffers sized for this problem.
        Matrix<double>* M = nullptr;
        A_sys->Init_Preconditioner(M, A_sys->n, P->len, P, o.mn, o.ns);
        size_t max_rows = static_cast<size_t>(A_sys->m) + 8;
        size_t max_cols = static_cast<size_t>(P->max_nnz) + static_cast<size_t>(o.mn) * o.ns + 8;
        if (max_cols > static_cast<size_t>(A_sys->n) + 8)
            max_cols = static_cast<size_t>(A_sys->n) + 8;
        // Largest |I_k|: rows reachable from the largest pattern column.
        size_t bs2 = static_cast<size_t>(A_sys->max_block_size) * A_sys->max_block_size;
        size_t ibound = static_cast<size_t>(A_sys->max_nnz) * max_cols;
        if (ibound > max_rows)
            ibound = max_rows;
        size_t idx_cap = (ibound > max_cols ? ibound : max_cols) + A_sys->max_nnz * max_cols + 16;
        if (idx_cap > max_rows + max_cols + 16)
            idx_cap = max_rows + max_cols + 16;
        size_t ahat = ibound * max_cols * bs2 + 16;
        size_t work = 256 * (max_cols * A_sys->max_block_size + 16);
        delete M->I_set;
        M->I_set = new Index_Set(static_cast<int>(idx_cap));
        delete M->J_set;
        M->J_set = new Index_Set(static_cast<int>(idx_cap));
        delete M->L_set;
        M->L_set = new Index_Set(static_cast<int>(idx_cap));
        delete M->U_Nls;
        M->U_Nls = new Index_Set(static_cast<int>(idx_cap));
        delete M->J_tilde_set;
        M->J_tilde_set = new Index_Set(static_cast<int>(idx_cap));
        replace_buffer(M->rhos, idx_cap);
        replace_buffer(M->first_index_set, idx_cap);
        replace_buffer(M->first_index_row, idx_cap);
        replace_buffer(M->A_Hat, ahat);
        replace_buffer(M->A_Hat_buffer, ahat);
        replace_buffer(M->mk_Hat, idx_cap * bs2);
        replace_buffer(M->mk_Hat_buffer, idx_cap * bs2);
        replace_buffer(M->bk_Hat, idx_cap * bs2);
        replace_buffer(M->residual_vals_b_buffer, idx_cap * bs2);
        replace_buffer(M->Tau_ptr, max_cols * A_sys->max_block_size + 16);
        replace_buffer(M->Work_qr_ptr, work);
        replace_buffer(M->Work_qt_ptr, work);
        const int hash_param = hash_sizes[o.hs];
        if (hash_param > 0)
            M->ht_M = new Hash_Table<double>(hash_param);

        // the columns to compute: all, a range, or a list
        std::vector<long> cols;
        const bool subset = o.col_lo >= 0 || o.col_file != nullptr;
        if (o.col_file) {
            FILE* cf = std::fopen(o.col_file, "r");
            if (!cf)
                throw std::runtime_error("cannot read the column file");
            long c = 0;
            while (std::fscanf(cf, "%ld", &c) == 1)
                if (c >= 0 && c < A_sys->n)
                    cols.push_back(c);
            std::fclose(cf);
        }
        else if (o.col_lo >= 0) {
            const long hi = o.col_hi > A_sys->n ? A_sys->n : o.col_hi;
            for (long c = o.col_lo; c < hi; c++)
                cols.push_back(c);
        }

        std::vector<double> rep_s;
        auto t0 = std::chrono::steady_clock::now();
        if (o.gpu) {
#ifdef MSPAI_GPU_SHIM
            if (subset || o.bs != 1)
                throw std::runtime_error("-gpu runs whole scalar setups");
            mspai_params extra;
            mspai_default_params(&extra);
            extra.cs = o.cs;
            extra.ch = o.ch;
            extra.qr = o.qr;
            extra.hs = o.hs;
            extra.prec = std::strcmp(o.gpu, "fp64") ? MSPAI_PREC_MIXED : MSPAI_PREC_FP64;
            mspai_b200_shim::Spai_GPU_Algorithm(A_sys, M, B, P, UP, o.ep, o.mn, o.ns,
                                                hash_param, o.um, o.pk, o.pm, /*count=*/1,
                                                o.vb, &extra);
#else
            throw std::runtime_error("-gpu: this driver was built without the drop-in");
#endif
        }
        else if (!subset) {
            alg->SPAI_Algorithm(A_sys, M, B, P, UP, o.ep, o.mn, o.ns, hash_param, o.um, o.pk,
                                o.pm, /*count=*/1, o.vb);
        }
        else {
            // Same per-run set-up as SPAI_Algorithm (src/Spai.imp:67-120), then
            // the reference's column routine on the listed columns.
            if (o.ns > 0)
                M->Precomputation_Column_Square_Inverses(A_sys);
            int bitvec_size = A_sys->m <= A_sys->n ? A_sys->n : A_sys->m;
            bitvec_size = (bitvec_size >> 5) + 1;
            std::memset(M->bitvec, 0, bitvec_size * sizeof(unsigned int));
            unsigned int* bitvec = M->bitvec;
            unsigned int* reset_vec = M->reset_vec;
            auto fn = Column_Access::fn();
            for (int r = 0; r < o.repeat; r++) {
                auto r0 = std::chrono::steady_clock::now();
                for (long col : cols)
                    (alg->*fn)(A_sys, M, B, P, UP, nullptr, static_cast<int>(col), o.ep, o.mn,
                               o.ns, M->ht_M, o.um, o.pk, o.pm, bitvec, reset_vec);
                rep_s.push_back(std::chrono::duration<double>(
                                    std::chrono::steady_clock::now() - r0).count());
            }
        }
        auto t1 = std::chrono::steady_clock::now();
        const double secs = rep_s.empty() ? std::chrono::duration<double>(t1 - t0).count()
                                          : rep_s.back();

        if (o.time_file) {
            FILE* f = std::fopen(o.time_file, "w");
            if (f) {
                std::fprintf(f, "{\"setup_s\": %.9f, \"columns\": %ld, \"rep_s\": [", secs,
                             subset ? static_cast<long>(cols.size()) : static_cast<long>(A_sys->n));
                for (size_t r = 0; r < rep_s.size(); r++)
                    std::fprintf(f, "%s%.9f", r ? ", " : "", rep_s[r]);
                std::fprintf(f, "]}\n");
                std::fclose(f);
            }
        }
        if (!subset) {
            if (A_sys->block_size != 1 || o.bs != 1) {
                Matrix<double>* S = M->Scalar_Matrix(0);
                S->Write_Matrix_To_File(o.out);
            }
            else {
                M->Write_Matrix_To_File(o.out);
            }
        }
        else {
            // The computed columns only, in the reference's output format, so
            // the subset can be compared column by column (block columns as
            // their scalar columns)
            Matrix<double>* S = (o.bs != 1) ? M->Scalar_Matrix(0) : M;
            const int bsz = (o.bs != 1) ? o.bs : 1;
            FILE* f = std::fopen(o.out, "w");
            if (!f)
                throw std::runtime_error("cannot write output");
            long nnz = 0;
            for (long c : cols)
                for (int q = 0; q < bsz; q++)
                    nnz += S->c_lines->len_cols[c * bsz + q];
            std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n%d %d %ld\n",
                         S->m, S->n, nnz);
            for (long c : cols)
                for (int q = 0; q < bsz; q++) {
                    const long sc = c * bsz + q;
                    for (int i = 0; i < S->c_lines->len_cols[sc]; i++) {
                        double v = S->c_lines->A[sc][i];
                        std::fprintf(f, "%d %ld%s%.13e\n", S->c_lines->col_idcs[sc][i] + 1,
                                     sc + 1, v < 0.0 ? " " : "  ", v);
                    }
                }
            std::fclose(f);
        }
        delete alg;
    }
    catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
