// mspai -- command-line front end of the B200 setup.
//
//   mspai <A.mtx> <pattern.mtx|-1|-2> <B.mtx|-1> [options]
//
// Positional arguments and options follow the reference's serial program
// (doc/mspai-1.2.pdf section 2.2-2.4; defaults src/Command_Line.cpp:192-225):
// -1 as pattern = diagonal start pattern, -2 = pattern of C; -1 as target =
// identity.  Options: -ep -mn -ns -hs -cs -qr -fg -um -ch -pk -pm -Ce -Be -rho
// -schur -up -bs -wp -vb -out.  Extra options of this implementation:
//   -prec fp64|mixed   arithmetic of the least-squares solves (mixed)
//   -refine k          FP64 refinement steps in mixed mode (2)
//   -batched 0|1       0 = plain per-column FP64 path (1)
//   -dev k             CUDA device (0)
// The preconditioner is written to -out (precond.mtx) in the reference's
// output format when -wp is 1 or -out is given.
#include "mspai_b200.h"
#include "mspai_b200_io.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

void usage()
{
    std::fprintf(stderr,
                 "usage: mspai <A.mtx> <pattern.mtx|-1|-2> <B.mtx|-1> [options]\n"
                 "  -ep x -mn k -ns k -hs k -cs k -qr k -fg x -um 0|1 -ch 0|1 -pk k -pm 0|1\n"
                 "  -Ce file -Be file -rho x -schur 0|1 -up file|1|2 -bs k -wp 0|1 -vb k\n"
                 "  -out file -prec fp64|mixed -refine k -batched 0|1 -dev k\n");
}

struct Owned {
    mspai_matrix m{};
    bool set = false;
    ~Owned()
    {
        if (set)
            mspai_matrix_free(&m);
    }
};

int read_or_die(const char* path, Owned& o)
{
    char msg[512];
    int rc = mspai_mm_read(path, &o.m, msg, sizeof(msg));
    if (rc != MSPAI_OK) {
        std::fprintf(stderr, "\n\tERROR:  %s\n", msg);
        return rc;
    }
    o.set = true;
    return MSPAI_OK;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 4 || !std::strcmp(argv[1], "-h") || !std::strcmp(argv[1], "-help")) {
        usage();
        return argc < 4 ? 1 : 0;
    }
    mspai_params prm;
    mspai_default_params(&prm);
    const char* a_file = argv[1];
    const char* p_arg = argv[2];
    const char* b_arg = argv[3];
    const char* ce_file = nullptr;
    const char* be_file = nullptr;
    const char* up_arg = nullptr;
    const char* out_file = "precond.mtx";
    int wp = 0, out_given = 0, dev = 0;
    for (int i = 4; i < argc; i += 2) {
        if (i + 1 >= argc) {
            usage();
            return 1;
        }
        const std::string k = argv[i];
        const char* v = argv[i + 1];
        if (k == "-ep") prm.ep = std::atof(v);
        else if (k == "-mn") prm.mn = std::atoi(v);
        else if (k == "-ns") prm.ns = std::atoi(v);
        else if (k == "-hs") prm.hs = std::atoi(v);
        else if (k == "-cs") prm.cs = std::atoi(v);
        else if (k == "-qr") prm.qr = std::atoi(v);
        else if (k == "-fg") prm.fg = std::atof(v);
        else if (k == "-um") prm.um = std::atoi(v);
        else if (k == "-ch") prm.ch = std::atoi(v);
        else if (k == "-pk") prm.pk = std::atoi(v);
        else if (k == "-pm") prm.pm = std::atoi(v);
        else if (k == "-schur") prm.schur = std::atoi(v);
        else if (k == "-rho") prm.rho = std::atof(v);
        else if (k == "-bs") prm.bs = std::atoi(v);
        else if (k == "-vb") prm.verbose = std::atoi(v);
        else if (k == "-wp") wp = std::atoi(v);
        else if (k == "-Ce") ce_file = v;
        else if (k == "-Be") be_file = v;
        else if (k == "-up") up_arg = v;
        else if (k == "-out") { out_file = v; out_given = 1; }
        else if (k == "-prec") prm.prec = !std::strcmp(v, "fp64") ? MSPAI_PREC_FP64 : MSPAI_PREC_MIXED;
        else if (k == "-refine") prm.refine = std::atoi(v);
        else if (k == "-batched") prm.batched = std::atoi(v);
        else if (k == "-dev") dev = std::atoi(v);
        else {
            std::fprintf(stderr, "unknown option %s\n", argv[i]);
            usage();
            return 1;
        }
    }
    prm.probing = ce_file != nullptr || be_file != nullptr;
    prm.target = std::strcmp(b_arg, "-1") == 0 ? 1 : 0;
    char msg[1024];
    int rc = mspai_validate_params(&prm, msg, sizeof(msg));
    if (rc != MSPAI_OK) {
        std::fprintf(stderr, "\n\t%s\n", msg);
        return rc;
    }
    Owned A, Ce, Be, C, B, P, UP, Bfile;
    if ((rc = read_or_die(a_file, A)) != MSPAI_OK)
        return rc;
    mspai_csc av = mspai_matrix_view(&A.m);
    if (ce_file && (rc = read_or_die(ce_file, Ce)) != MSPAI_OK)
        return rc;
    if (be_file && (rc = read_or_die(be_file, Be)) != MSPAI_OK)
        return rc;
    mspai_csc cev = mspai_matrix_view(&Ce.m), bev = mspai_matrix_view(&Be.m);
    rc = mspai_probing_assemble(&av, ce_file ? &cev : nullptr, be_file ? &bev : nullptr, prm.rho,
                                &C.m, &B.m, msg, sizeof(msg));
    if (rc != MSPAI_OK) {
        std::fprintf(stderr, "\n\tERROR:  %s\n", msg);
        return rc;
    }
    C.set = B.set = true;
    mspai_csc cv = mspai_matrix_view(&C.m);
    mspai_csc bv = mspai_matrix_view(&B.m);
    const mspai_csc* Bptr = prm.probing ? &bv : nullptr;
    if (!prm.target) {
        if ((rc = read_or_die(b_arg, Bfile)) != MSPAI_OK)
            return rc;
        bv = mspai_matrix_view(&Bfile.m);
        Bptr = &bv;
    }
    if (prm.bs > 1 && (!std::strcmp(p_arg, "-1") || !std::strcmp(p_arg, "-2"))) {
        // block start pattern over the n / bs block columns (a pattern file is
        // read as such a block pattern)
        rc = mspai_block_pattern_generate(&cv, prm.bs, !std::strcmp(p_arg, "-1") ? 1 : 2, &P.m);
        if (rc != MSPAI_OK) {
            std::fprintf(stderr, "\n\tERROR:  block size %d does not divide n = %d\n", prm.bs,
                         cv.ncols);
            return rc;
        }
        P.set = true;
    }
    else if (!std::strcmp(p_arg, "-1") || !std::strcmp(p_arg, "-2")) {
        rc = mspai_pattern_generate(&cv, !std::strcmp(p_arg, "-1") ? 1 : 2, &P.m);
        if (rc != MSPAI_OK)
            return rc;
        P.set = true;
    }
    else if ((rc = read_or_die(p_arg, P)) != MSPAI_OK) {
        return rc;
    }
    mspai_csc pv = mspai_matrix_view(&P.m);
    pv.values = nullptr;
    const mspai_csc* UPptr = nullptr;
    mspai_csc upv{};
    if (up_arg && prm.bs > 1) {
        std::fprintf(stderr, "\n\tERROR:  an upper pattern (-up) with -bs %d is not supported\n",
                     prm.bs);
        return MSPAI_ERR_PARAM;
    }
    if (up_arg) {
        if (!std::strcmp(up_arg, "1") || !std::strcmp(up_arg, "2")) {
            rc = mspai_pattern_generate(&cv, up_arg[0] == '1' ? 1 : 2, &UP.m);
            if (rc != MSPAI_OK)
                return rc;
            UP.set = true;
        }
        else if ((rc = read_or_die(up_arg, UP)) != MSPAI_OK) {
            return rc;
        }
        upv = mspai_matrix_view(&UP.m);
        upv.values = nullptr;
        UPptr = &upv;
    }
    mspai_handle* h = nullptr;
    rc = mspai_create(&h, dev, nullptr);
    if (rc != MSPAI_OK) {
        std::fprintf(stderr, "\n\tERROR:  no usable CUDA device (%d)\n", rc);
        return rc;
    }
    const auto t0 = std::chrono::steady_clock::now();
    rc = mspai_setup(h, &cv, nullptr, Bptr, &pv, UPptr, &prm);
    const auto t1 = std::chrono::steady_clock::now();
    if (rc != MSPAI_OK) {
        std::fprintf(stderr, "\n\tERROR:  %s\n", mspai_last_error(h));
        mspai_free(h);
        return rc;
    }
    mspai_stats st{};
    mspai_get_stats(h, &st);
    if (prm.verbose)
        std::printf("\t* Computing SPAI...\t\t\t %.6f [sec] (device %.6f)\n",
                    std::chrono::duration<double>(t1 - t0).count(), st.setup_ms * 1e-3);
    if (wp || out_given) {
        int64_t nnz = 0;
        mspai_result_nnz(h, &nnz);
        std::vector<int64_t> mp(static_cast<size_t>(cv.ncols) + 1);
        std::vector<int32_t> mi(static_cast<size_t>(nnz > 0 ? nnz : 1));
        std::vector<double> mv(static_cast<size_t>(nnz > 0 ? nnz : 1));
        rc = mspai_result_copy(h, mp.data(), mi.data(), mv.data(), MSPAI_MEM_HOST);
        if (rc == MSPAI_OK) {
            mspai_csc mvw{cv.ncols, cv.ncols, nnz, mp.data(), mi.data(), mv.data(), MSPAI_MEM_HOST};
            rc = mspai_mm_write(out_file, &mvw, msg, sizeof(msg));
            if (rc != MSPAI_OK)
                std::fprintf(stderr, "\n\tERROR:  %s\n", msg);
        }
    }
    mspai_free(h);
    return rc;
}
