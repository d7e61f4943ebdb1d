// Host engine behind the C ABI of include/mspai_b200.h.
//
// mspai_setup replaces Spai<double>::SPAI_Algorithm (reference
// src/Spai.imp:33-191): it stages the inputs in device memory, plans and bins
// the columns by problem size, runs the bucket kernels, and assembles M's CSC
// on the device.  Everything a setup allocates is owned by the handle and
// reused by the next setup of the same or a smaller size.
#include "mspai_b200.h"
#include "host_util.h"
#include "spai_kernels.h"
#include "spai_solve.cuh"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

using mspai::BucketRule;
using mspai::Caps;
using mspai::Output;
using mspai::Problem;

constexpr int kBuckets = 3;    // size buckets of the planning kernel
constexpr int kKernels = 4;    // solver launches per setup (timed separately)
constexpr int kLists = 4;      // work lists: buckets + the overflow lists
// Arena of the fixed-pattern solver's second launch (one CTA per SM): the
// largest dynamic shared memory a CTA may have beside the solver's static part.
constexpr int kFixedArenaLarge = 212 * 1024;
// Mixed precision solves a bucket whose largest |J_k| (after the pattern
// updates) is at most this in FP64 directly: the FP32 QR saves nothing on such
// sizes, and the refinement would add two passes over the column's entries.
constexpr int kMixedFp64MaxN = 32;

// A device buffer that grows on demand.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t want)
    {
        if (want <= bytes && p)
            return cudaSuccess;
        if (p)
            cudaFree(p);
        p = nullptr;
        bytes = 0;
        size_t alloc = std::max<size_t>(want, 256);
        cudaError_t e = cudaMalloc(&p, alloc);
        if (e == cudaSuccess)
            bytes = alloc;
        return e;
    }
    void release()
    {
        if (p)
            cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    template <class T>
    T* as() const
    {
        return static_cast<T*>(p);
    }
};

}  // namespace

struct mspai_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::string err;
    // staged inputs
    DevBuf cptr, cidx, cval, rptr, rcol, bptr, bidx, bval, pptr, pidx, upptr, upidx;
    // planning
    DevBuf E, nk, lists, counters, scan_tmp, cap_len, cap_ptr;
    // outputs
    DevBuf oidx, oval, olen, res, steps, status, work;
    DevBuf mptr, midx, mval;  // final M
    DevBuf scratch;
    DevBuf vflag;  // device input checks
    DevBuf ax, ay; // host vectors of mspai_apply
    // row structure of the result for mspai_apply (built on first use)
    DevBuf tptr, tcol, tval, tkeys, tperm0, tperm1, tcnt, ttemp;
    bool rows_valid = false;
    DevBuf rkeys, rslot_rep, rslot_of, rrep;  // reuse table
    DevBuf rglob;  // per-CTA areas for R of the fixed-pattern solver
    DevBuf rstore, roff;  // R of every column (keep_factors), packed by columns
    DevBuf rhash;         // structure digest of C, P, B (device accumulator)
    bool r_valid = false;
    int r_elem = 8;
    unsigned long long r_hash = 0;  // digest of the setup whose R is kept
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t evb[2 * kKernels] = {};
    // result description
    int n = 0;
    int64_t nnz_m = 0;
    bool have_result = false;
    bool fixed_pattern = true;
    const int64_t* res_ptr = nullptr;
    const int32_t* res_idx = nullptr;
    const double* res_val = nullptr;
    mspai_stats stats{};
    mspai_params last_params{};
    int64_t launches = 0;
    int nprob = 0;  // problem columns of the last setup (n / bs)
    size_t smem_budget = 48 * 1024;  // shared-memory area of each CTA solver (4 per SM)
    int fixed_arena = 107 * 1024;    // arena of the fixed-pattern solver's first launch (2 CTAs per SM)
    int fixed_arena_large = kFixedArenaLarge;  // ... and of its second launch
    int warp_emax = 64;              // tiny bucket: entries of C(:, J_k) ...
    int warp_nmax = 16;              // ... and |J_k|
    int64_t w_smem_bytes = 96 * 1024;  // general solver: folded matrices up to this in smem
    int warp_emax_adaptive = 256;    // adaptive tiny bucket (warp per column, global slots)
    int warp_nmax_adaptive = 32;
    bool used_fixed = false;         // the last setup ran the fixed-pattern solver
    int64_t list_len[kLists] = {};   // columns listed per work list in the last setup
};

static int set_err(mspai_handle* h, int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (h)
        h->err = buf;
    return code;
}

#define CUDA_TRY(h, expr)                                                                        \
    do {                                                                                         \
        cudaError_t _e = (expr);                                                                 \
        if (_e != cudaSuccess)                                                                   \
            return set_err((h), _e == cudaErrorMemoryAllocation ? MSPAI_ERR_ALLOC : MSPAI_ERR_CUDA, \
                           "%s: %s (%s:%d)", #expr, cudaGetErrorString(_e), __FILE__, __LINE__); \
    } while (0)

// Stages an array on the device: borrows device pointers, copies host ones.
template <class T>
static cudaError_t stage(DevBuf& buf, const T* src, size_t count, int mem, cudaStream_t st,
                         const T** out)
{
    if (src == nullptr || count == 0) {
        *out = nullptr;
        if (count == 0 && src != nullptr) {
            cudaError_t e = buf.ensure(sizeof(T));
            *out = buf.as<T>();
            return e;
        }
        return cudaSuccess;
    }
    if (mem == MSPAI_MEM_DEVICE) {
        *out = src;
        return cudaSuccess;
    }
    cudaError_t e = buf.ensure(count * sizeof(T));
    if (e != cudaSuccess)
        return e;
    e = cudaMemcpyAsync(buf.p, src, count * sizeof(T), cudaMemcpyHostToDevice, st);
    *out = buf.as<T>();
    return e;
}

template <class T>
static cudaError_t fetch(std::vector<T>& dst, const T* src, size_t count, int mem, cudaStream_t st)
{
    dst.resize(count);
    if (count == 0)
        return cudaSuccess;
    if (mem == MSPAI_MEM_HOST) {
        std::memcpy(dst.data(), src, count * sizeof(T));
        return cudaSuccess;
    }
    cudaError_t e = cudaMemcpyAsync(dst.data(), src, count * sizeof(T), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess)
        return e;
    return cudaStreamSynchronize(st);
}

extern "C" {

const char* mspai_version(void) { return "mspai_b200 0.1"; }

int mspai_create(mspai_handle** out, int32_t device, void* stream)
{
    if (!out)
        return MSPAI_ERR_PARAM;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        cudaGetLastError();
        return MSPAI_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= count)
        return MSPAI_ERR_NO_DEVICE;
    mspai_handle* h = new (std::nothrow) mspai_handle();
    if (!h)
        return MSPAI_ERR_ALLOC;
    h->device = device;
    if (cudaSetDevice(device) != cudaSuccess) {
        delete h;
        return MSPAI_ERR_CUDA;
    }
    if (stream) {
        h->stream = static_cast<cudaStream_t>(stream);
    }
    else {
        if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete h;
            return MSPAI_ERR_CUDA;
        }
        h->own_stream = true;
    }
    cudaEventCreate(&h->ev0);
    cudaEventCreate(&h->ev1);
    for (auto& e : h->evb)
        cudaEventCreate(&e);
    if (const char* kb = std::getenv("MSPAI_SMEM_KB")) {
        const long v = std::atol(kb);
        if (v >= 16 && v <= 220)
            h->smem_budget = static_cast<size_t>(v) * 1024;
    }
    // arenas of the fixed-pattern solver's two launches (KB); small values send
    // columns down the overflow chain (used by the tests of that chain)
    if (const char* kb = std::getenv("MSPAI_FIXED_ARENA_KB")) {
        const long v = std::atol(kb);
        if (v >= 1 && v <= 216)
            h->fixed_arena = static_cast<int>(v) * 1024;
    }
    if (const char* kb = std::getenv("MSPAI_FIXED_ARENA_LARGE_KB")) {
        const long v = std::atol(kb);
        if (v >= 1 && v <= 216)
            h->fixed_arena_large = static_cast<int>(v) * 1024;
    }
    *out = h;
    return MSPAI_OK;
}

void mspai_free(mspai_handle* h)
{
    if (!h)
        return;
    cudaSetDevice(h->device);
    if (h->stream)
        cudaStreamSynchronize(h->stream);
    DevBuf* bufs[] = {&h->cptr, &h->cidx, &h->cval, &h->rptr, &h->rcol, &h->bptr, &h->bidx,
                      &h->bval, &h->pptr, &h->pidx, &h->upptr, &h->upidx, &h->E, &h->nk,
                      &h->lists, &h->counters, &h->scan_tmp, &h->cap_len, &h->cap_ptr, &h->oidx,
                      &h->oval, &h->olen, &h->res, &h->steps, &h->status, &h->work, &h->mptr,
                      &h->midx, &h->mval, &h->scratch, &h->vflag, &h->ax, &h->ay,
                      &h->rkeys, &h->rslot_rep, &h->rslot_of, &h->rrep, &h->tptr, &h->tcol,
                      &h->tval, &h->tkeys, &h->tperm0, &h->tperm1, &h->tcnt, &h->ttemp,
                      &h->rglob};
    for (DevBuf* b : bufs)
        b->release();
    if (h->ev0)
        cudaEventDestroy(h->ev0);
    if (h->ev1)
        cudaEventDestroy(h->ev1);
    for (auto& e : h->evb)
        if (e)
            cudaEventDestroy(e);
    if (h->own_stream && h->stream)
        cudaStreamDestroy(h->stream);
    delete h;
}

const char* mspai_last_error(mspai_handle* h)
{
    return h ? h->err.c_str() : "null handle";
}

static int check_csc(mspai_handle* h, const mspai_csc* m, const char* name, bool need_values)
{
    if (!m->colptr || (m->nnz > 0 && !m->rowidx))
        return set_err(h, MSPAI_ERR_INPUT, "%s: missing arrays", name);
    if (need_values && m->nnz > 0 && !m->values)
        return set_err(h, MSPAI_ERR_INPUT, "%s: missing values", name);
    if (m->nrows < 0 || m->ncols < 0 || m->nnz < 0)
        return set_err(h, MSPAI_ERR_INPUT, "%s: negative size", name);
    if (m->mem != MSPAI_MEM_HOST && m->mem != MSPAI_MEM_DEVICE)
        return set_err(h, MSPAI_ERR_INPUT, "%s: bad memory kind", name);
    // the structure itself (pointers, row range, sorted unique rows) is
    // checked on the device after staging, for host and device inputs alike
    return MSPAI_OK;
}

// A staged CSC structure to check on the device.
struct CscCheck {
    const char* name;
    const int64_t* ptr;
    const int32_t* idx;
    int ncols, nrows;
    int64_t nnz;
    bool nonempty;  // every column needs an entry (C: src/Read_mm_Matrix.cpp:745-751)
};

// Runs the device checks of `k` staged structures and reports the first error
// of the first failing one with the messages of the host checks.  No kernel
// that indexes with these structures runs before this returns MSPAI_OK.
static int validate_on_device(mspai_handle* h, const CscCheck* cs, int k, cudaStream_t st)
{
    CUDA_TRY(h, h->vflag.ensure(sizeof(int32_t) * 4 * k));
    int32_t* vf = h->vflag.as<int32_t>();
    CUDA_TRY(h, cudaMemsetAsync(vf, 0, sizeof(int32_t) * 4 * k, st));
    for (int i = 0; i < k; i++)
        CUDA_TRY(h, mspai::launch_validate_csc(cs[i].ptr, cs[i].idx, cs[i].ncols, cs[i].nrows,
                                               cs[i].nnz, cs[i].nonempty, vf + 4 * i, st));
    int32_t hv[4 * 8] = {};
    CUDA_TRY(h, cudaMemcpyAsync(hv, vf, sizeof(int32_t) * 4 * k, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    for (int i = 0; i < k; i++) {
        const int kind = hv[4 * i], c = hv[4 * i + 1], r = hv[4 * i + 2];
        const char* nm = cs[i].name;
        switch (kind) {
        case 0: break;
        case 1:
            return set_err(h, MSPAI_ERR_INPUT, "%s: column pointers do not match nnz", nm);
        case 2: return set_err(h, MSPAI_ERR_INPUT, "%s: column pointers decrease", nm);
        case 3:
            return set_err(h, MSPAI_ERR_INPUT, "%s: row index %d out of range in column %d", nm,
                           r, c);
        case 4:
            return set_err(h, MSPAI_ERR_INPUT, "%s: row indices not sorted/unique in column %d",
                           nm, c);
        default:
            return set_err(h, MSPAI_ERR_INPUT, "Matrix is singular: column %d of C is empty", c);
        }
    }
    return MSPAI_OK;
}

int mspai_setup(mspai_handle* h, const mspai_csc* C, const mspai_csc* C_rows, const mspai_csc* B,
                const mspai_csc* P, const mspai_csc* UP, const mspai_params* prm)
{
    if (!h)
        return MSPAI_ERR_STATE;
    h->err.clear();
    h->have_result = false;
    h->rows_valid = false;
    if (!C || !P || !prm)
        return set_err(h, MSPAI_ERR_PARAM, "C, P and params are required");
    char msg[1024];
    int rc = mspai_validate_params(prm, msg, sizeof(msg));
    if (rc != MSPAI_OK)
        return set_err(h, rc, "%s", msg);
    const int n = C->ncols;
    const int bs = prm->bs;
    if (prm->schur)
        return set_err(h, MSPAI_ERR_PARAM,
                       "Schur probing (-schur 1) is not supported by this setup: its target "
                       "[0; I; rho Be] and the n x N_p pattern are not built");
    if (bs > mspai::kMaxBlockSize)
        return set_err(h, MSPAI_ERR_PARAM, "block size %d not supported (1..%d)", bs,
                       mspai::kMaxBlockSize);
    if (n % bs != 0)
        return set_err(h, MSPAI_ERR_INPUT,
                       "block size %d does not divide the %d columns (constant blocks only)", bs,
                       n);
    const int nprob = n / bs;  // problem columns: scalar columns or block columns
    // column range of this call (sharding over GPUs): [col_lo, col_hi)
    const int col_lo = prm->col_begin;
    const int col_hi = prm->col_end > 0 ? prm->col_end : nprob;
    if (col_lo < 0 || col_hi > nprob || col_lo > col_hi)
        return set_err(h, MSPAI_ERR_PARAM, "column range [%d, %d) outside [0, %d)", col_lo,
                       col_hi, nprob);
    const bool partial = col_lo > 0 || col_hi < nprob;
    if ((rc = check_csc(h, C, "C", true)) != MSPAI_OK)
        return rc;
    if ((rc = check_csc(h, P, "P", false)) != MSPAI_OK)
        return rc;
    if (C->nrows < n)
        return set_err(h, MSPAI_ERR_INPUT, "C has fewer rows (%d) than columns (%d)", C->nrows, n);
    if (P->ncols != nprob || P->nrows != nprob)
        return set_err(h, MSPAI_ERR_INPUT, "%spattern must be %d x %d", bs > 1 ? "block " : "",
                       nprob, nprob);
    if (B) {
        if ((rc = check_csc(h, B, "B", true)) != MSPAI_OK)
            return rc;
        if (B->ncols != n || B->nrows != C->nrows)
            return set_err(h, MSPAI_ERR_INPUT, "target must be %d x %d", C->nrows, n);
    }
    if (UP) {
        if ((rc = check_csc(h, UP, "UP", false)) != MSPAI_OK)
            return rc;
        if (UP->ncols != n || UP->nrows != n)
            return set_err(h, MSPAI_ERR_INPUT, "upper pattern must be %d x %d", n, n);
    }
    CUDA_TRY(h, cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    const bool adaptive = prm->ns > 0 && prm->mn > 0;
    h->fixed_pattern = !adaptive;
    h->n = n;

    // ---- stage inputs
    Problem pb{};
    pb.n = n;
    pb.nrows = C->nrows;
    CUDA_TRY(h, stage(h->cptr, C->colptr, n + 1, C->mem, st, &pb.cptr));
    CUDA_TRY(h, stage(h->cidx, C->rowidx, C->nnz, C->mem, st, &pb.cidx));
    CUDA_TRY(h, stage(h->cval, C->values, C->nnz, C->mem, st, &pb.cval));
    CUDA_TRY(h, stage(h->pptr, P->colptr, nprob + 1, P->mem, st, &pb.pptr));
    CUDA_TRY(h, stage(h->pidx, P->rowidx, P->nnz, P->mem, st, &pb.pidx));
    if (B) {
        CUDA_TRY(h, stage(h->bptr, B->colptr, n + 1, B->mem, st, &pb.bptr));
        CUDA_TRY(h, stage(h->bidx, B->rowidx, B->nnz, B->mem, st, &pb.bidx));
        CUDA_TRY(h, stage(h->bval, B->values, B->nnz, B->mem, st, &pb.bval));
    }
    if (UP) {
        CUDA_TRY(h, stage(h->upptr, UP->colptr, n + 1, UP->mem, st, &pb.upptr));
        CUDA_TRY(h, stage(h->upidx, UP->rowidx, UP->nnz, UP->mem, st, &pb.upidx));
    }
    int check_launches = 0;
    {
        CscCheck cs[4];
        int k = 0;
        cs[k++] = CscCheck{"C", pb.cptr, pb.cidx, n, C->nrows, C->nnz, true};
        cs[k++] = CscCheck{"P", pb.pptr, pb.pidx, nprob, nprob, P->nnz, false};
        if (B)
            cs[k++] = CscCheck{"B", pb.bptr, pb.bidx, n, C->nrows, B->nnz, false};
        if (UP)
            cs[k++] = CscCheck{"UP", pb.upptr, pb.upidx, n, n, UP->nnz, false};
        if ((rc = validate_on_device(h, cs, k, st)) != MSPAI_OK)
            return rc;
        check_launches = k;
    }
    int max_row_nnz = 0, max_col_nnz = 0;
    if (adaptive) {
        std::vector<int64_t> rp;
        std::vector<int32_t> rc2;
        if (C_rows) {
            if ((rc = check_csc(h, C_rows, "C_rows", false)) != MSPAI_OK)
                return rc;
            if (C_rows->ncols < n || C_rows->nrows != n)
                return set_err(h, MSPAI_ERR_INPUT, "C_rows must be the %d x (>= %d) CSC of C^T",
                               n, n);
            CUDA_TRY(h, stage(h->rptr, C_rows->colptr, C_rows->ncols + 1, C_rows->mem, st, &pb.rptr));
            CUDA_TRY(h, stage(h->rcol, C_rows->rowidx, C_rows->nnz, C_rows->mem, st, &pb.rcol));
            {
                const CscCheck cr{"C_rows", pb.rptr, pb.rcol, C_rows->ncols, C_rows->nrows,
                                  C_rows->nnz, false};
                if ((rc = validate_on_device(h, &cr, 1, st)) != MSPAI_OK)
                    return rc;
                check_launches++;
            }
            CUDA_TRY(h, fetch(rp, C_rows->colptr, C_rows->ncols + 1, C_rows->mem, st));
        }
        else {
            // the row structure of C on the device: a stable radix sort of the
            // entries by row keeps each row's columns ascending; rows below n
            // are a prefix of it (the probing rows come last)
            const int nr = C->nrows;
            const int64_t nz = C->nnz;
            const size_t tb = mspai::rows_build_temp_bytes(nz, nr);
            CUDA_TRY(h, h->rptr.ensure(sizeof(int64_t) * (static_cast<size_t>(nr) + 1)));
            CUDA_TRY(h, h->rcol.ensure(sizeof(int32_t) * std::max<int64_t>(nz, 1)));
            CUDA_TRY(h, h->tkeys.ensure(sizeof(int32_t) * std::max<int64_t>(nz, 1)));
            CUDA_TRY(h, h->tperm0.ensure(sizeof(int32_t) * std::max<int64_t>(nz, 1)));
            CUDA_TRY(h, h->tperm1.ensure(sizeof(int32_t) * std::max<int64_t>(nz, 1)));
            CUDA_TRY(h, h->tcnt.ensure(sizeof(int32_t) * std::max(nr, 1)));
            CUDA_TRY(h, h->ttemp.ensure(std::max<size_t>(tb, 16)));
            CUDA_TRY(h, h->scan_tmp.ensure(sizeof(int64_t) * ((nr + 1023) / 1024 + 2)));
            h->launches += 7;
            CUDA_TRY(h, mspai::launch_build_rows(
                            pb.cptr, pb.cidx, nullptr, n, nr, nz, h->rptr.as<int64_t>(),
                            h->rcol.as<int32_t>(), nullptr, h->tkeys.as<int32_t>(),
                            h->tperm0.as<int32_t>(), h->tperm1.as<int32_t>(),
                            h->tcnt.as<int32_t>(), h->scan_tmp.as<int64_t>(), h->ttemp.p,
                            h->ttemp.bytes, st));
            pb.rptr = h->rptr.as<int64_t>();
            pb.rcol = h->rcol.as<int32_t>();
            CUDA_TRY(h, h->counters.ensure(64 * sizeof(int32_t)));
            int32_t* mx = h->counters.as<int32_t>() + 17;
            h->launches++;
            CUDA_TRY(h, mspai::launch_max_len(pb.rptr, n, mx, st));
            CUDA_TRY(h, cudaMemcpyAsync(&max_row_nnz, mx, sizeof(int32_t), cudaMemcpyDeviceToHost,
                                        st));
            CUDA_TRY(h, cudaStreamSynchronize(st));
        }
        for (size_t i = 0; i + 1 < rp.size(); i++)
            max_row_nnz = std::max<int>(max_row_nnz, static_cast<int>(rp[i + 1] - rp[i]));
    }
    pb.bs = bs;
    pb.ep = prm->ep;
    pb.mn = prm->mn;
    pb.ns = adaptive ? prm->ns : 0;
    pb.um = prm->um;
    const bool mixed = prm->prec == MSPAI_PREC_MIXED && prm->batched;
    // QR updates (-qr > 0) keep and extend each column's factorization across
    // the pattern steps (batched scalar adaptive setups)
    pb.qru = (prm->qr > 0 && adaptive && bs == 1 && prm->batched) ? 1 : 0;
    pb.refine = mixed ? std::max(0, prm->refine) : 0;
    const int elem = mixed ? 4 : 8;

    // ---- time the device part of the setup
    h->launches = check_launches;  // the input checks ran on the device too
    CUDA_TRY(h, cudaEventRecord(h->ev0, st));

    // max column nnz of C (growth bound of the entry count)
    CUDA_TRY(h, h->counters.ensure(64 * sizeof(int32_t)));
    int32_t* dcnt = h->counters.as<int32_t>();
    h->launches++;
    CUDA_TRY(h, mspai::launch_max_len(pb.cptr, n, dcnt + 16, st));
    CUDA_TRY(h, cudaMemcpyAsync(&max_col_nnz, dcnt + 16, sizeof(int32_t), cudaMemcpyDeviceToHost, st));

    // ---- output capacity
    Output out{};
    const int grow_n = adaptive ? prm->mn * prm->ns : 0;
    CUDA_TRY(h, h->olen.ensure(sizeof(int32_t) * std::max(n, 1)));
    CUDA_TRY(h, h->res.ensure(sizeof(double) * std::max(n, 1)));
    CUDA_TRY(h, h->steps.ensure(sizeof(int32_t) * std::max(n, 1)));
    CUDA_TRY(h, h->status.ensure(sizeof(int32_t) * std::max(n, 1)));
    CUDA_TRY(h, h->work.ensure(sizeof(double) * 3 * std::max(n, 1)));
    CUDA_TRY(h, cudaMemsetAsync(h->work.p, 0, sizeof(double) * 3 * std::max(n, 1), st));
    CUDA_TRY(h, h->scan_tmp.ensure(sizeof(int64_t) * ((n + 1023) / 1024 + 2)));
    int64_t cap_total = P->nnz;
    const bool compact = adaptive || bs > 1;  // M's pattern differs from P's
    h->fixed_pattern = !compact;
    if (compact) {
        CUDA_TRY(h, h->cap_len.ensure(sizeof(int32_t) * std::max(n, 1)));
        CUDA_TRY(h, h->cap_ptr.ensure(sizeof(int64_t) * (n + 1)));
        h->launches++;
        CUDA_TRY(h, mspai::launch_capacity_len(pb.pptr, n, bs, grow_n, h->cap_len.as<int32_t>(),
                                               st));
        h->launches += 4;
        CUDA_TRY(h, mspai::launch_scan_lengths(h->cap_len.as<int32_t>(), n, h->cap_ptr.as<int64_t>(),
                                               h->scan_tmp.as<int64_t>(), st));
        cap_total = (P->nnz + static_cast<int64_t>(grow_n) * nprob) * bs * bs;
        CUDA_TRY(h, h->oidx.ensure(sizeof(int32_t) * std::max<int64_t>(cap_total, 1)));
        out.optr = h->cap_ptr.as<int64_t>();
        out.oidx = h->oidx.as<int32_t>();
        out.write_idx = 1;
    }
    else {
        out.optr = pb.pptr;
        out.oidx = nullptr;
        out.write_idx = 0;
    }
    CUDA_TRY(h, h->oval.ensure(sizeof(double) * std::max<int64_t>(cap_total, 1)));
    out.oval = h->oval.as<double>();
    if (partial) {
        // columns outside the range stay empty (zero values, length 0)
        CUDA_TRY(h, cudaMemsetAsync(h->oval.p, 0, sizeof(double) * std::max<int64_t>(cap_total, 1),
                                    st));
        CUDA_TRY(h, cudaMemsetAsync(h->olen.p, 0, sizeof(int32_t) * std::max(n, 1), st));
        CUDA_TRY(h, cudaMemsetAsync(h->res.p, 0, sizeof(double) * std::max(n, 1), st));
        CUDA_TRY(h, cudaMemsetAsync(h->steps.p, 0, sizeof(int32_t) * std::max(n, 1), st));
        CUDA_TRY(h, cudaMemsetAsync(h->status.p, 0, sizeof(int32_t) * std::max(n, 1), st));
    }
    out.olen = h->olen.as<int32_t>();
    out.res = h->res.as<double>();
    out.steps = h->steps.as<int32_t>();
    out.status = h->status.as<int32_t>();
    out.work = h->work.as<double>();
    // ---- the columns' triangular factors for the adjoint and for re-setups
    // (fixed scalar patterns)
    bool reuse_now = false;
    unsigned long long shash = 0;
    if (prm->keep_factors && !compact) {
        // digest of the structures of C, P and B: a re-setup from the kept
        // factors needs the structure of the setup that kept them
        CUDA_TRY(h, h->rhash.ensure(sizeof(unsigned long long)));
        auto* acc = h->rhash.as<unsigned long long>();
        CUDA_TRY(h, cudaMemsetAsync(acc, 0, sizeof(unsigned long long), st));
        h->launches += pb.bptr ? 3 : 2;
        CUDA_TRY(h, mspai::launch_structure_hash(pb.cptr, pb.cidx, n, C->nnz,
                                                 0x436f6c756d6e73ull, acc, st));
        CUDA_TRY(h, mspai::launch_structure_hash(pb.pptr, pb.pidx, nprob, P->nnz,
                                                 0x5061747465726eull, acc, st));
        if (pb.bptr)
            CUDA_TRY(h, mspai::launch_structure_hash(pb.bptr, pb.bidx, n, B->nnz,
                                                     0x546172676574ull, acc, st));
        CUDA_TRY(h, cudaMemcpyAsync(&shash, acc, sizeof(shash), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(h, cudaStreamSynchronize(st));
        shash ^= (static_cast<unsigned long long>(C->nrows) << 32) ^
                 static_cast<unsigned long long>(elem);
        reuse_now = prm->reuse_factors > 0 && h->r_valid && h->r_hash == shash &&
                    h->r_elem == elem && !partial && prm->batched;
    }
    h->r_valid = false;
    if (prm->keep_factors && !compact) {
        CUDA_TRY(h, h->cap_len.ensure(sizeof(int32_t) * std::max(n, 1)));
        CUDA_TRY(h, h->roff.ensure(sizeof(int64_t) * (n + 1)));
        h->launches += 5;
        CUDA_TRY(h, mspai::launch_tri_len(pb.pptr, n, h->cap_len.as<int32_t>(), st));
        CUDA_TRY(h, mspai::launch_scan_lengths(h->cap_len.as<int32_t>(), n, h->roff.as<int64_t>(),
                                               h->scan_tmp.as<int64_t>(), st));
        int64_t rtotal = 0;
        CUDA_TRY(h, cudaMemcpyAsync(&rtotal, h->roff.as<int64_t>() + n, sizeof(int64_t),
                                    cudaMemcpyDeviceToHost, st));
        CUDA_TRY(h, cudaStreamSynchronize(st));
        CUDA_TRY(h, h->rstore.ensure(static_cast<size_t>(elem) * std::max<int64_t>(rtotal, 1)));
        out.rstore = h->rstore.p;
        out.roff = h->roff.as<int64_t>();
        h->r_elem = elem;
        if (reuse_now) {
            // M's previous values are still in oval (same structure, no range)
            out.reuse_steps = prm->reuse_factors;
            out.reuse_count = h->counters.as<int32_t>() + 40;
            CUDA_TRY(h, cudaMemsetAsync(out.reuse_count, 0, sizeof(int32_t), st));
        }
    }

    // ---- plan and bucket
    CUDA_TRY(h, h->E.ensure(sizeof(int32_t) * std::max(nprob, 1)));
    CUDA_TRY(h, h->nk.ensure(sizeof(int32_t) * std::max(nprob, 1)));
    CUDA_TRY(h, h->lists.ensure(sizeof(int32_t) * static_cast<size_t>(kLists) *
                                std::max(nprob, 1)));
    h->launches++;
    CUDA_TRY(h, mspai::launch_plan(pb.cptr, pb.pptr, pb.pidx, nprob, bs, h->E.as<int32_t>(),
                                   h->nk.as<int32_t>(), st));
    // ---- reuse of identical problems (-cs / -ch): fixed scalar and block
    // patterns (not with keep_factors: a reused column has no factor of its own)
    const bool reuse = (prm->cs > 0 || prm->ch > 0) && !adaptive && prm->batched &&
                       !partial && !prm->keep_factors;
    int32_t* drep = nullptr;
    if (reuse) {
        const int max_keys = prm->cs > 0 ? prm->cs : nprob;
        const size_t slots = mspai::reuse_table_slots(nprob, max_keys);
        CUDA_TRY(h, h->rkeys.ensure(sizeof(uint64_t) * slots));
        CUDA_TRY(h, h->rslot_rep.ensure(sizeof(int32_t) * slots));
        CUDA_TRY(h, h->rslot_of.ensure(sizeof(int32_t) * std::max(nprob, 1)));
        CUDA_TRY(h, h->rrep.ensure(sizeof(int32_t) * std::max(nprob, 1)));
        mspai::ReuseTable tab{};
        tab.keys = h->rkeys.as<uint64_t>();
        tab.rep_of_slot = h->rslot_rep.as<int32_t>();
        tab.slot_of = h->rslot_of.as<int32_t>();
        tab.nkeys = dcnt + 20;
        tab.mask = static_cast<uint32_t>(slots - 1);
        tab.max_keys = max_keys;
        drep = h->rrep.as<int32_t>();
        h->launches += 2;
        CUDA_TRY(h, mspai::launch_reuse_keys(pb, nprob, tab, drep, dcnt + 21, st));
    }
    CUDA_TRY(h, cudaStreamSynchronize(st));  // max_col_nnz is on the host now
    BucketRule rule{};
    rule.rep = drep;
    rule.lo = col_lo;
    rule.hi = col_hi;
    rule.single_bucket = prm->batched ? -1 : 2;
    // tiny bucket: a warp per column (adaptive scalar setups too, with the
    // slots in global memory; not with the QR-update state)
    rule.allow_warp = (bs > 1 || pb.qru) ? 0 : 1;
    rule.warp_emax = adaptive ? h->warp_emax_adaptive : h->warp_emax;
    rule.warp_nmax = adaptive ? h->warp_nmax_adaptive : h->warp_nmax;
    // fixed scalar patterns: every column beyond the warp bucket goes to the
    // fixed-pattern solver (bucket 1), which sizes its arrays per column
    const bool use_fixed = !adaptive && bs == 1 && prm->batched && !pb.qru;
    rule.smem_w_bytes = use_fixed ? (int64_t(1) << 62) : h->w_smem_bytes;
    rule.elem_bytes = elem;
    rule.grow_n = grow_n * bs;
    rule.grow_e = adaptive ? grow_n * bs * max_col_nnz : 0;
    CUDA_TRY(h, cudaMemsetAsync(dcnt, 0, sizeof(int32_t) * 16, st));
    h->launches++;
    CUDA_TRY(h, mspai::launch_bucket(h->E.as<int32_t>(), h->nk.as<int32_t>(), nprob, rule, dcnt,
                                     dcnt + 4, dcnt + 8, h->lists.as<int32_t>(), st));
    int32_t hc[16];
    CUDA_TRY(h, cudaMemcpyAsync(hc, dcnt, sizeof(hc), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));

    // ---- bucket kernels
    for (int k = 0; k < kKernels; k++) {
        h->stats.bucket_columns[k] = 0;
        h->stats.kernel_ms[k] = 0.0;
    }
    for (int k = 0; k < kLists; k++)
        h->list_len[k] = 0;
    bool timed[kKernels] = {false, false, false, false};
    h->used_fixed = use_fixed;
    // general CTA solver over `count` listed columns with the given caps
    auto run_cta = [&](int b, const Caps& cap, int32_t* list, int count, int32_t* counter,
                       size_t wsm_budget, int elem_b, const Problem& pbb) -> int {
        int grid = 0;
        size_t wsm = std::min<size_t>(mspai::w_bytes(cap, elem_b), wsm_budget);
        if (!prm->batched)
            wsm = 0;  // the plain path keeps W in global memory, unblocked
        const size_t need = mspai::cta_scratch_needed(elem_b, cap, count, wsm);
        CUDA_TRY(h, h->scratch.ensure(need));
        if (adaptive)  // the candidate bit vectors of the slots start cleared
            CUDA_TRY(h, cudaMemsetAsync(h->scratch.p, 0, need, st));
        CUDA_TRY(h, cudaMemsetAsync(counter, 0, sizeof(int32_t), st));
        h->launches++;
        CUDA_TRY(h, mspai::launch_cta_solve(elem_b, wsm, prm->batched != 0, pbb, cap, out, list,
                                            count, counter, h->scratch.as<char>(),
                                            h->scratch.bytes, st, &grid));
        (void)b;
        return MSPAI_OK;
    };
    for (int b = 0; b < kBuckets; b++) {
        const int count = hc[b];
        if (!(use_fixed && b == 2))  // with the fixed-pattern solver list 2 is its overflow
            h->list_len[b] = count;
        if (count == 0)
            continue;
        Caps cap{};
        cap.emax = std::max(1, hc[4 + b]);
        cap.nmax = std::max(1, hc[8 + b]);
        cap.lsort = mspai::next_pow2(cap.emax);
        cap.mwmax = cap.emax / 2 + cap.nmax;
        cap.nrhs = bs;
        // unique candidates: at most the problem columns, at most the row
        // structure entries of L's rows
        cap.cmax = adaptive ? static_cast<int>(std::min<int64_t>(
                                  nprob, static_cast<int64_t>(cap.emax + 1) * bs *
                                             std::max(1, max_row_nnz)))
                            : 0;
        cap.lcand = adaptive ? mspai::next_pow2(cap.cmax) : 0;
        cap.nbmap = adaptive ? (nprob + 31) / 32 : 0;
        cap.qru = pb.qru;
        if (static_cast<int64_t>(cap.emax) >= mspai::kMaxEntries)
            return set_err(h, MSPAI_ERR_CAPACITY, "a column touches %d entries of C (max %d)",
                           cap.emax, mspai::kMaxEntries - 1);
        int32_t* list = h->lists.as<int32_t>() + static_cast<size_t>(b) * nprob;
        int32_t* counter = dcnt + 12 + b;
        CUDA_TRY(h, cudaMemsetAsync(counter, 0, sizeof(int32_t), st));
        int grid = 0;
        // small problems in mixed mode: FP64 without refinement (not when R
        // is kept: its store has one element type)
        const bool fp64_bucket = mixed && !out.rstore && cap.nmax <= kMixedFp64MaxN;
        const int elem_b = fp64_bucket ? 8 : elem;
        Problem pbb = pb;
        if (fp64_bucket)
            pbb.refine = 0;
        bool use_warp = (b == 0);
        const bool warp_global =
            use_warp && (adaptive || mspai::warp_slot_bytes(cap, elem_b) *
                                             (mspai::kWarpKernelThreads / 32) > 200 * 1024);
        if (warp_global) {
            const size_t need = mspai::warp_global_scratch_bytes(cap, elem_b, count);
            CUDA_TRY(h, h->scratch.ensure(need));
            if (adaptive)  // the candidate bit vectors of the slots start cleared
                CUDA_TRY(h, cudaMemsetAsync(h->scratch.p, 0, need, st));
            CUDA_TRY(h, cudaEventRecord(h->evb[0], st));
            h->launches++;
            CUDA_TRY(h, mspai::launch_warp_solve_global(elem_b, pbb, cap, out, list, count,
                                                        counter, h->scratch.as<char>(),
                                                        h->scratch.bytes, st, &grid));
            CUDA_TRY(h, cudaEventRecord(h->evb[1], st));
            timed[0] = true;
            h->stats.bucket_columns[0] = count;
        }
        else if (use_warp) {
            CUDA_TRY(h, cudaEventRecord(h->evb[0], st));
            h->launches++;
            CUDA_TRY(h, mspai::launch_warp_solve(elem_b, pbb, cap, out, list, count, counter, st,
                                                 &grid));
            CUDA_TRY(h, cudaEventRecord(h->evb[1], st));
            timed[0] = true;
            h->stats.bucket_columns[0] = count;
        }
        else if (b == 1 && use_fixed) {
            // fixed-pattern solver: launch A (tuned arena) over the bucket, its
            // overflow through launch B (the largest arena), what is left
            // through the general solver
            int32_t* ovf_a = h->lists.as<int32_t>() + static_cast<size_t>(2) * nprob;
            int32_t* ovf_b = h->lists.as<int32_t>() + static_cast<size_t>(3) * nprob;
            int32_t* cnt = dcnt + 24;  // [0] overflow A, [1] overflow B, [2] queue B
            CUDA_TRY(h, cudaMemsetAsync(cnt, 0, 3 * sizeof(int32_t), st));
            const int64_t relems = mspai::fixed_r_elems(cap.nmax);
            const int grid_max = std::max(mspai::fixed_max_grid(h->fixed_arena),
                                          mspai::fixed_max_grid(h->fixed_arena_large));
            CUDA_TRY(h, h->rglob.ensure(static_cast<size_t>(grid_max) * relems * elem));
            CUDA_TRY(h, cudaEventRecord(h->evb[2], st));
            h->launches++;
            CUDA_TRY(h, mspai::launch_fixed_solve(elem, h->fixed_arena, pb, out, list, nullptr,
                                                  count, counter, ovf_a, cnt, h->rglob.p, relems,
                                                  grid_max, st, &grid));
            CUDA_TRY(h, cudaEventRecord(h->evb[3], st));
            CUDA_TRY(h, cudaEventRecord(h->evb[4], st));
            h->launches++;
            CUDA_TRY(h, mspai::launch_fixed_solve(elem, h->fixed_arena_large, pb, out, ovf_a, cnt, 0,
                                                  cnt + 2, ovf_b, cnt + 1, h->rglob.p, relems,
                                                  grid_max, st, &grid));
            CUDA_TRY(h, cudaEventRecord(h->evb[5], st));
            timed[1] = timed[2] = true;
            int32_t ho[2] = {0, 0};
            CUDA_TRY(h, cudaMemcpyAsync(ho, cnt, sizeof(ho), cudaMemcpyDeviceToHost, st));
            CUDA_TRY(h, cudaStreamSynchronize(st));
            h->list_len[2] = ho[0];
            h->list_len[3] = ho[1];
            h->stats.bucket_columns[1] = count - ho[0];
            h->stats.bucket_columns[2] = ho[0] - ho[1];
            h->stats.bucket_columns[3] = ho[1];
            if (ho[1] > 0) {
                CUDA_TRY(h, cudaEventRecord(h->evb[6], st));
                const int rc2 = run_cta(3, cap, ovf_b, ho[1], dcnt + 15, 48 * 1024, elem, pb);
                if (rc2 != MSPAI_OK)
                    return rc2;
                CUDA_TRY(h, cudaEventRecord(h->evb[7], st));
                timed[3] = true;
            }
        }
        else {
            CUDA_TRY(h, cudaEventRecord(h->evb[2 * b], st));
            const int rc2 = run_cta(b, cap, list, count, counter, h->smem_budget, elem_b, pbb);
            if (rc2 != MSPAI_OK)
                return rc2;
            CUDA_TRY(h, cudaEventRecord(h->evb[2 * b + 1], st));
            timed[b] = true;
            h->stats.bucket_columns[b] = count;
        }
    }

    if (reuse) {
        h->launches++;
        CUDA_TRY(h, mspai::launch_reuse_copy(drep, nprob, bs, out, st));
    }

    // ---- assemble M
    if (compact) {
        CUDA_TRY(h, h->mptr.ensure(sizeof(int64_t) * (n + 1)));
        h->launches += 4;
        CUDA_TRY(h, mspai::launch_scan_lengths(out.olen, n, h->mptr.as<int64_t>(),
                                               h->scan_tmp.as<int64_t>(), st));
        int64_t nnz = 0;
        CUDA_TRY(h, cudaMemcpyAsync(&nnz, h->mptr.as<int64_t>() + n, sizeof(int64_t),
                                    cudaMemcpyDeviceToHost, st));
        CUDA_TRY(h, cudaStreamSynchronize(st));
        CUDA_TRY(h, h->midx.ensure(sizeof(int32_t) * std::max<int64_t>(nnz, 1)));
        CUDA_TRY(h, h->mval.ensure(sizeof(double) * std::max<int64_t>(nnz, 1)));
        h->launches++;
    CUDA_TRY(h, mspai::launch_compact(out.optr, out.oidx, out.oval, h->mptr.as<int64_t>(),
                                          h->midx.as<int32_t>(), h->mval.as<double>(), n, st));
        h->nnz_m = nnz;
        h->res_ptr = h->mptr.as<int64_t>();
        h->res_idx = h->midx.as<int32_t>();
        h->res_val = h->mval.as<double>();
    }
    else {
        h->nnz_m = P->nnz;
        h->res_ptr = pb.pptr;
        h->res_idx = pb.pidx;
        h->res_val = out.oval;
        if (P->mem == MSPAI_MEM_HOST) {
            // keep the structure alive in the handle's buffers (already staged)
        }
        else {
            // borrowed device pattern: copy so the result outlives the call
            CUDA_TRY(h, h->mptr.ensure(sizeof(int64_t) * (n + 1)));
            CUDA_TRY(h, h->midx.ensure(sizeof(int32_t) * std::max<int64_t>(P->nnz, 1)));
            CUDA_TRY(h, cudaMemcpyAsync(h->mptr.p, pb.pptr, sizeof(int64_t) * (n + 1),
                                        cudaMemcpyDeviceToDevice, st));
            if (P->nnz > 0)
                CUDA_TRY(h, cudaMemcpyAsync(h->midx.p, pb.pidx, sizeof(int32_t) * P->nnz,
                                            cudaMemcpyDeviceToDevice, st));
            h->res_ptr = h->mptr.as<int64_t>();
            h->res_idx = h->midx.as<int32_t>();
        }
    }
    CUDA_TRY(h, cudaEventRecord(h->ev1, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    CUDA_TRY(h, cudaGetLastError());
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->stats.setup_ms = ms;
    for (int k = 0; k < kKernels; k++) {
        if (timed[k]) {
            float kms = 0.f;
            cudaEventElapsedTime(&kms, h->evb[2 * k], h->evb[2 * k + 1]);
            h->stats.kernel_ms[k] = kms;
        }
    }
    h->stats.reused_columns = 0;
    if (reuse) {
        int32_t nre = 0;
        CUDA_TRY(h, cudaMemcpy(&nre, dcnt + 21, sizeof(int32_t), cudaMemcpyDeviceToHost));
        h->stats.reused_columns = nre;
    }
    h->stats.columns = static_cast<int64_t>(col_hi - col_lo) * bs;
    h->nprob = nprob;
    h->stats.nnz_m = h->nnz_m;
    h->stats.kernel_launches = h->launches;
    h->last_params = *prm;
    h->have_result = true;
    h->r_valid = out.rstore != nullptr;
    h->r_hash = shash;
    h->stats.factor_reuse_columns = 0;
    if (out.reuse_count) {
        int32_t nr = 0;
        CUDA_TRY(h, cudaMemcpy(&nr, out.reuse_count, sizeof(int32_t), cudaMemcpyDeviceToHost));
        h->stats.factor_reuse_columns = nr;
    }
    return MSPAI_OK;
}

int mspai_result_nnz(mspai_handle* h, int64_t* nnz)
{
    if (!h || !h->have_result)
        return h ? set_err(h, MSPAI_ERR_STATE, "no setup result") : MSPAI_ERR_STATE;
    *nnz = h->nnz_m;
    return MSPAI_OK;
}

int mspai_tune(mspai_handle* h, const mspai_csc* C, const mspai_csc* C_rows, const mspai_csc* B,
               const mspai_csc* P, const mspai_csc* UP, const mspai_params* prm,
               int32_t sample_cols, int32_t* smem_kb_out)
{
    if (!h || !C || !P || !prm)
        return h ? set_err(h, MSPAI_ERR_PARAM, "C, P and params are required") : MSPAI_ERR_STATE;
    // candidates: the per-CTA shared-memory area, which sets the CTAs per SM
    // of the solver (48 KB: 4, 32 KB: 6, 24 KB: 8) and how much of each
    // column's work (key merge, packed R) stays in shared memory
    static const int kCandidates[] = {48, 32, 24};
    const int nprob = P->ncols;
    const int cols = std::max(1, std::min<int>(sample_cols > 0 ? sample_cols : 20000, nprob));
    mspai_params q = *prm;
    q.col_begin = 0;
    q.col_end = cols;
    int best = kCandidates[0];
    double best_ms = 1e300;
    for (int kb : kCandidates) {
        h->smem_budget = static_cast<size_t>(kb) * 1024;
        double ms = 0.0;
        for (int rep = 0; rep < 2; rep++) {  // the first run warms up
            const int rc = mspai_setup(h, C, C_rows, B, P, UP, &q);
            if (rc != MSPAI_OK)
                return rc;
            ms = h->stats.setup_ms;
        }
        if (ms < best_ms) {
            best_ms = ms;
            best = kb;
        }
    }
    h->smem_budget = static_cast<size_t>(best) * 1024;
    h->have_result = false;  // the sample runs are not a result
    h->r_valid = false;
    if (smem_kb_out)
        *smem_kb_out = best;
    return MSPAI_OK;
}

int mspai_get_tuning(mspai_handle* h, mspai_tuning* t)
{
    if (!h || !t)
        return h ? set_err(h, MSPAI_ERR_PARAM, "tuning is required") : MSPAI_ERR_STATE;
    t->smem_kb = static_cast<int32_t>(h->smem_budget / 1024);
    t->fixed_arena_kb = h->fixed_arena / 1024;
    t->fixed_arena_large_kb = h->fixed_arena_large / 1024;
    t->warp_emax = h->warp_emax;
    t->warp_nmax = h->warp_nmax;
    t->w_smem_kb = static_cast<int32_t>(h->w_smem_bytes / 1024);
    t->warp_emax_adaptive = h->warp_emax_adaptive;
    t->warp_nmax_adaptive = h->warp_nmax_adaptive;
    return MSPAI_OK;
}

int mspai_set_tuning(mspai_handle* h, const mspai_tuning* t)
{
    if (!h || !t)
        return h ? set_err(h, MSPAI_ERR_PARAM, "tuning is required") : MSPAI_ERR_STATE;
    auto in = [](int v, int lo, int hi) { return v >= lo && v <= hi; };
    if (!in(t->smem_kb, 16, 220) || !in(t->fixed_arena_kb, 8, 107) ||
        !in(t->fixed_arena_large_kb, 8, 212) || !in(t->warp_emax, 16, 256) ||
        !in(t->warp_nmax, 4, 32) || !in(t->w_smem_kb, 16, 220) ||
        !in(t->warp_emax_adaptive, 16, 4096) || !in(t->warp_nmax_adaptive, 4, 64))
        return set_err(h, MSPAI_ERR_PARAM,
                       "tuning out of range: smem_kb 16..220, fixed_arena_kb 8..107, "
                       "fixed_arena_large_kb 8..212, warp_emax 16..256, warp_nmax 4..32, "
                       "w_smem_kb 16..220, warp_emax_adaptive 16..4096, "
                       "warp_nmax_adaptive 4..64");
    h->smem_budget = static_cast<size_t>(t->smem_kb) * 1024;
    h->fixed_arena = t->fixed_arena_kb * 1024;
    h->fixed_arena_large = t->fixed_arena_large_kb * 1024;
    h->warp_emax = t->warp_emax;
    h->warp_nmax = t->warp_nmax;
    h->w_smem_bytes = static_cast<int64_t>(t->w_smem_kb) * 1024;
    h->warp_emax_adaptive = t->warp_emax_adaptive;
    h->warp_nmax_adaptive = t->warp_nmax_adaptive;
    return MSPAI_OK;
}

int mspai_apply(mspai_handle* h, const double* x, double* y, int32_t mem)
{
    if (!h || !h->have_result)
        return h ? set_err(h, MSPAI_ERR_STATE, "no setup result") : MSPAI_ERR_STATE;
    if (!x || !y)
        return set_err(h, MSPAI_ERR_PARAM, "x and y are required");
    CUDA_TRY(h, cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    const int n = h->n;
    const double* dx = x;
    double* dy = y;
    if (mem == MSPAI_MEM_HOST) {
        CUDA_TRY(h, h->ax.ensure(sizeof(double) * std::max(n, 1)));
        CUDA_TRY(h, h->ay.ensure(sizeof(double) * std::max(n, 1)));
        CUDA_TRY(h, cudaMemcpyAsync(h->ax.p, x, sizeof(double) * n, cudaMemcpyHostToDevice, st));
        dx = h->ax.as<double>();
        dy = h->ay.as<double>();
    }
    if (!h->rows_valid) {
        const int64_t nnz = h->nnz_m;
        if (nnz >= (int64_t(1) << 31))
            return set_err(h, MSPAI_ERR_CAPACITY, "M has too many nonzeros for mspai_apply");
        const size_t nz = static_cast<size_t>(std::max<int64_t>(nnz, 1));
        const size_t tb = std::max<size_t>(mspai::rows_build_temp_bytes(nnz, n), 16);
        CUDA_TRY(h, h->tptr.ensure(sizeof(int64_t) * (n + 1)));
        CUDA_TRY(h, h->tcol.ensure(sizeof(int32_t) * nz));
        CUDA_TRY(h, h->tval.ensure(sizeof(double) * nz));
        CUDA_TRY(h, h->tkeys.ensure(sizeof(int32_t) * nz));
        CUDA_TRY(h, h->tperm0.ensure(sizeof(int32_t) * nz));
        CUDA_TRY(h, h->tperm1.ensure(sizeof(int32_t) * nz));
        CUDA_TRY(h, h->tcnt.ensure(sizeof(int32_t) * std::max(n, 1)));
        CUDA_TRY(h, h->ttemp.ensure(tb));
        CUDA_TRY(h, h->scan_tmp.ensure(sizeof(int64_t) * ((n + 1023) / 1024 + 2)));
        CUDA_TRY(h, mspai::launch_build_rows(
                        h->res_ptr, h->res_idx, h->res_val, n, n, nnz, h->tptr.as<int64_t>(),
                        h->tcol.as<int32_t>(), h->tval.as<double>(), h->tkeys.as<int32_t>(),
                        h->tperm0.as<int32_t>(), h->tperm1.as<int32_t>(), h->tcnt.as<int32_t>(),
                        h->scan_tmp.as<int64_t>(), h->ttemp.p, h->ttemp.bytes, st));
        h->rows_valid = true;
    }
    CUDA_TRY(h, mspai::launch_csr_gather(h->tptr.as<int64_t>(), h->tcol.as<int32_t>(),
                                         h->tval.as<double>(), n, dx, dy, st));
    if (mem == MSPAI_MEM_HOST)
        CUDA_TRY(h, cudaMemcpyAsync(y, dy, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    return MSPAI_OK;
}

int mspai_result_copy(mspai_handle* h, int64_t* colptr, int32_t* rowidx, double* values,
                      int32_t mem)
{
    if (!h || !h->have_result)
        return h ? set_err(h, MSPAI_ERR_STATE, "no setup result") : MSPAI_ERR_STATE;
    CUDA_TRY(h, cudaSetDevice(h->device));
    const cudaMemcpyKind k = mem == MSPAI_MEM_DEVICE ? cudaMemcpyDeviceToDevice
                                                     : cudaMemcpyDeviceToHost;
    cudaStream_t st = h->stream;
    if (colptr)
        CUDA_TRY(h, cudaMemcpyAsync(colptr, h->res_ptr, sizeof(int64_t) * (h->n + 1), k, st));
    if (rowidx && h->nnz_m > 0)
        CUDA_TRY(h, cudaMemcpyAsync(rowidx, h->res_idx, sizeof(int32_t) * h->nnz_m, k, st));
    if (values && h->nnz_m > 0)
        CUDA_TRY(h, cudaMemcpyAsync(values, h->res_val, sizeof(double) * h->nnz_m, k, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    return MSPAI_OK;
}

int mspai_column_info(mspai_handle* h, double* resnorm, int32_t* steps, int32_t* status)
{
    if (!h || !h->have_result)
        return h ? set_err(h, MSPAI_ERR_STATE, "no setup result") : MSPAI_ERR_STATE;
    CUDA_TRY(h, cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    if (resnorm)
        CUDA_TRY(h, cudaMemcpyAsync(resnorm, h->res.p, sizeof(double) * h->n,
                                    cudaMemcpyDeviceToHost, st));
    if (steps)
        CUDA_TRY(h, cudaMemcpyAsync(steps, h->steps.p, sizeof(int32_t) * h->n,
                                    cudaMemcpyDeviceToHost, st));
    if (status)
        CUDA_TRY(h, cudaMemcpyAsync(status, h->status.p, sizeof(int32_t) * h->n,
                                    cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    return MSPAI_OK;
}

int mspai_get_stats(mspai_handle* h, mspai_stats* s)
{
    if (!h || !h->have_result)
        return h ? set_err(h, MSPAI_ERR_STATE, "no setup result") : MSPAI_ERR_STATE;
    CUDA_TRY(h, cudaSetDevice(h->device));
    std::vector<double> work(3 * static_cast<size_t>(h->n));
    std::vector<int32_t> steps(h->n), status(h->n);
    if (h->n > 0) {
        CUDA_TRY(h, cudaMemcpyAsync(work.data(), h->work.p, sizeof(double) * work.size(),
                                    cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(h, cudaMemcpyAsync(steps.data(), h->steps.p, sizeof(int32_t) * h->n,
                                    cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(h, cudaMemcpyAsync(status.data(), h->status.p, sizeof(int32_t) * h->n,
                                    cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    }
    double fl = 0.0, fld = 0.0, by = 0.0;
    int64_t solves = 0, sing = 0, capc = 0;
    // algorithmic flops per solver launch: the columns of its work list that
    // it solved (a fixed-pattern launch passes the columns it could not hold
    // on to the next list)
    for (int b = 0; b < 4; b++)
        h->stats.bucket_flops[b] = 0.0;
    if (h->nprob > 0 && h->lists.p) {
        std::vector<int32_t> lists(static_cast<size_t>(kLists) * h->nprob);
        CUDA_TRY(h, cudaMemcpy(lists.data(), h->lists.p, sizeof(int32_t) * lists.size(),
                               cudaMemcpyDeviceToHost));
        double sums[kLists] = {0.0, 0.0, 0.0, 0.0};
        for (int b = 0; b < kLists; b++)
            for (int64_t t = 0; t < h->list_len[b]; t++)
                sums[b] += work[3 * static_cast<size_t>(lists[b * static_cast<size_t>(h->nprob) + t])];
        if (h->used_fixed) {
            h->stats.bucket_flops[0] = sums[0];
            h->stats.bucket_flops[1] = sums[1] - sums[2];
            h->stats.bucket_flops[2] = sums[2] - sums[3];
            h->stats.bucket_flops[3] = sums[3];
        }
        else {
            for (int b = 0; b < kBuckets; b++)
                h->stats.bucket_flops[b] = sums[b];
        }
    }
    for (int c = 0; c < h->n; c++) {
        fl += work[3 * c];
        fld += work[3 * c + 1];
        by += work[3 * c + 2];
        solves += steps[c];
        sing += status[c] == MSPAI_COL_SINGULAR;
        capc += status[c] == MSPAI_COL_CAPACITY;
    }
    h->stats.flops = fl;
    h->stats.flops_dense = fld;
    h->stats.gather_bytes = by;
    h->stats.ls_solves = solves;
    h->stats.singular_columns = sing;
    h->stats.capacity_columns = capc;
    *s = h->stats;
    return MSPAI_OK;
}

}  // extern "C"

extern "C" int mspai_adjoint(mspai_handle* h, const mspai_csc* C, const mspai_csc* B,
                             const double* gbar_values, double* dC_values, double* dB_values,
                             double* loss, int32_t mem)
{
    return mspai_adjoint_weighted(h, C, B, gbar_values, 1.0, dC_values, dB_values, loss, mem);
}

extern "C" int mspai_adjoint_weighted(mspai_handle* h, const mspai_csc* C, const mspai_csc* B,
                                      const double* gbar_values, double residual_weight,
                                      double* dC_values, double* dB_values, double* loss,
                                      int32_t mem)
{
    if (!h || !h->have_result)
        return h ? set_err(h, MSPAI_ERR_STATE, "no setup result") : MSPAI_ERR_STATE;
    const int bs = std::max(1, h->last_params.bs);
    if (gbar_values && bs != 1)
        return set_err(h, MSPAI_ERR_PARAM,
                       "gbar needs a scalar setup (bs = 1): block columns have no gbar term");
    if (!C || !dC_values)
        return set_err(h, MSPAI_ERR_PARAM, "C and dC are required");
    if (!std::isfinite(residual_weight))
        return set_err(h, MSPAI_ERR_PARAM, "the residual weight must be finite");
    if (C->ncols != h->n)
        return set_err(h, MSPAI_ERR_INPUT, "C does not match the last setup");
    if (B && (B->ncols != h->n || B->nrows != C->nrows))
        return set_err(h, MSPAI_ERR_INPUT, "B does not match C");
    CUDA_TRY(h, cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    const int n = h->n;
    const int nprob = h->nprob;
    Problem pb{};
    pb.n = n;
    pb.nrows = C->nrows;
    CUDA_TRY(h, stage(h->cptr, C->colptr, n + 1, C->mem, st, &pb.cptr));
    CUDA_TRY(h, stage(h->cidx, C->rowidx, C->nnz, C->mem, st, &pb.cidx));
    CUDA_TRY(h, stage(h->cval, C->values, C->nnz, C->mem, st, &pb.cval));
    if (B) {
        CUDA_TRY(h, stage(h->bptr, B->colptr, n + 1, B->mem, st, &pb.bptr));
        CUDA_TRY(h, stage(h->bidx, B->rowidx, B->nnz, B->mem, st, &pb.bidx));
        CUDA_TRY(h, stage(h->bval, B->values, B->nnz, B->mem, st, &pb.bval));
    }
    pb.bs = bs;
    mspai::AdjointIO io{};
    io.mptr = h->res_ptr;
    io.midx = h->res_idx;
    io.mval = h->res_val;
    io.wres = residual_weight;
    DevBuf gbuf, dcbuf, dbbuf, lossbuf, cnt;
    if (gbar_values) {
        const double* gp = nullptr;
        CUDA_TRY(h, stage(gbuf, gbar_values, static_cast<size_t>(h->nnz_m), mem, st, &gp));
        io.gbar = gp;
        if (h->r_valid) {
            io.rstore = h->rstore.p;
            io.roff = h->roff.as<int64_t>();
            io.r_elem = h->r_elem;
        }
    }
    if (mem == MSPAI_MEM_DEVICE) {
        io.dC = dC_values;
        io.dB = B ? dB_values : nullptr;
    }
    else {
        CUDA_TRY(h, dcbuf.ensure(sizeof(double) * std::max<int64_t>(C->nnz, 1)));
        io.dC = dcbuf.as<double>();
        if (B && dB_values) {
            CUDA_TRY(h, dbbuf.ensure(sizeof(double) * std::max<int64_t>(B->nnz, 1)));
            io.dB = dbbuf.as<double>();
        }
    }
    CUDA_TRY(h, cudaMemsetAsync(io.dC, 0, sizeof(double) * C->nnz, st));
    if (io.dB)  // entries of columns outside the setup's range stay zero
        CUDA_TRY(h, cudaMemsetAsync(io.dB, 0, sizeof(double) * B->nnz, st));
    CUDA_TRY(h, lossbuf.ensure(sizeof(double) * std::max(nprob, 1)));
    io.loss = lossbuf.as<double>();
    CUDA_TRY(h, cudaMemsetAsync(io.loss, 0, sizeof(double) * std::max(nprob, 1), st));
    // sizes: entries and pattern length of each problem column at the result's pattern
    CUDA_TRY(h, cnt.ensure(64 * sizeof(int32_t)));
    int32_t* dcnt = cnt.as<int32_t>();
    CUDA_TRY(h, cudaMemsetAsync(dcnt, 0, 64 * sizeof(int32_t), st));
    CUDA_TRY(h, h->E.ensure(sizeof(int32_t) * std::max(nprob, 1)));
    CUDA_TRY(h, h->nk.ensure(sizeof(int32_t) * std::max(nprob, 1)));
    CUDA_TRY(h, h->lists.ensure(sizeof(int32_t) * 3 * static_cast<size_t>(std::max(nprob, 1))));
    h->launches++;
    CUDA_TRY(h, mspai::launch_adjoint_plan(pb.cptr, io.mptr, io.midx, nprob, bs,
                                           h->E.as<int32_t>(), h->nk.as<int32_t>(), st));
    // the columns of the last setup
    const int alo = h->last_params.col_begin;
    const int ahi = h->last_params.col_end > 0 ? h->last_params.col_end : nprob;
    BucketRule rule{};
    rule.single_bucket = 0;
    rule.elem_bytes = 8;
    rule.lo = alo;
    rule.hi = ahi;
    h->launches++;
    CUDA_TRY(h, mspai::launch_bucket(h->E.as<int32_t>(), h->nk.as<int32_t>(), nprob, rule, dcnt,
                                     dcnt + 4, dcnt + 8, h->lists.as<int32_t>(), st));
    int32_t hc[16];
    CUDA_TRY(h, cudaMemcpyAsync(hc, dcnt, sizeof(hc), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(h, cudaStreamSynchronize(st));
    Caps cap{};
    cap.emax = std::max(1, hc[4]);
    cap.nmax = std::max(1, hc[8]);
    cap.lsort = mspai::next_pow2(cap.emax);
    cap.mwmax = cap.emax / 2 + cap.nmax;
    cap.cmax = cap.emax;  // q = C lambda is kept in the rho[] area
    cap.lcand = 0;
    cap.nrhs = bs;
    cap.nbmap = 0;
    const bool warp = cap.emax <= 64 && cap.nmax <= 16;
    const size_t need = mspai::adjoint_scratch_bytes(cap, nprob, warp);
    CUDA_TRY(h, h->scratch.ensure(need));
    CUDA_TRY(h, cudaMemsetAsync(dcnt + 20, 0, sizeof(int32_t), st));
    h->launches++;
    CUDA_TRY(h, mspai::launch_adjoint(pb, cap, io, alo, ahi, warp, h->scratch.as<char>(),
                                      h->scratch.bytes, dcnt + 20, st));
    std::vector<double> hl(nprob);
    if (nprob > 0)
        CUDA_TRY(h, cudaMemcpyAsync(hl.data(), io.loss, sizeof(double) * nprob,
                                    cudaMemcpyDeviceToHost, st));
    if (mem == MSPAI_MEM_HOST) {
        CUDA_TRY(h, cudaMemcpyAsync(dC_values, io.dC, sizeof(double) * C->nnz,
                                    cudaMemcpyDeviceToHost, st));
        if (io.dB)
            CUDA_TRY(h, cudaMemcpyAsync(dB_values, io.dB, sizeof(double) * B->nnz,
                                        cudaMemcpyDeviceToHost, st));
    }
    CUDA_TRY(h, cudaStreamSynchronize(st));
    CUDA_TRY(h, cudaGetLastError());
    if (loss) {
        // compensated (Neumaier) sum: the columns' losses are often nearly
        // equal, and a plain running sum lets their rounding errors add up
        double s = 0.0, comp = 0.0;
        for (double v : hl) {
            const double t = s + v;
            comp += std::fabs(s) >= std::fabs(v) ? (s - t) + v : (v - t) + s;
            s = t;
        }
        *loss = s + comp;
    }
    gbuf.release();
    dcbuf.release();
    dbbuf.release();
    lossbuf.release();
    cnt.release();
    return MSPAI_OK;
}
